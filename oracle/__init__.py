"""CPU oracle for TAL-SH's tensor-algebra path (TEST INFRASTRUCTURE ONLY).

Thin ctypes wrapper over ``libtalsh_oracle.so`` (built from
``talsh_oracle.cpp`` by ``oracle/Makefile``), a C++ restatement of the
reference's CP-TAL path in ``TALSH/tensor_algebra_cpu.F90``.  Only the tests,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs use it, as the checker
or the timed CPU baseline; the product package never imports it.

Arrays are numpy arrays in TAL-SH's "dlf" layout: a tensor with extents
``dims`` (dimension 1 fastest) is a flat array of ``prod(dims)`` elements, or
any array whose Fortran-order flattening is that.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

R4, R8, C4, C8 = 4, 8, 14, 18
NP_DTYPE = {R4: np.float32, R8: np.float64, C4: np.complex64, C8: np.complex128}
DTK_OF = {np.dtype(v): k for k, v in NP_DTYPE.items()}

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libtalsh_oracle.so")
_lib = None

OPENBLAS_CANDIDATES = [
    "/opt/prime-rl/.venv/lib/python3.12/site-packages/scipy.libs/libscipy_openblas-5f890258.so",
]


def build(force: bool = False) -> str:
    """Compile the oracle library with ``make`` (g++, OpenMP, -ffp-contract=off)."""
    if force or not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "talsh_oracle.cpp"))):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        ip = C.POINTER(C.c_int)
        L.orc_parse_pattern.argtypes = [C.c_char_p, ip, ip, ip, ip, ip]
        L.orc_contr_permutations.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, ip, C.c_int,
                                             ip, ip, ip, ip, ip, ip]
        L.orc_permute.argtypes = [C.c_int, C.c_int, ip, ip, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.orc_permute_blocked.argtypes = [C.c_int, C.c_int, ip, ip, C.c_void_p, C.c_void_p, C.c_int]
        L.orc_add.argtypes = [C.c_int, C.c_int64, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                              C.c_int, C.c_int, C.c_int]
        L.orc_tensor_add.argtypes = [ip, C.c_int, C.c_int, ip, C.c_void_p, C.c_void_p, C.c_double,
                                     C.c_double, C.c_int, C.c_int]
        L.orc_scale.argtypes = [C.c_int, C.c_int64, C.c_void_p, C.c_double, C.c_double]
        L.orc_init.argtypes = [C.c_int, C.c_int64, C.c_void_p, C.c_double, C.c_double]
        L.orc_norm.argtypes = [C.c_int, C.c_int64, C.c_void_p, C.c_int]
        L.orc_norm.restype = C.c_double
        L.orc_fill_uniform.argtypes = [C.c_int64, C.c_uint64, C.c_double, C.c_double, C.c_void_p, C.c_int]
        L.orc_dd_dot_batch.argtypes = [C.c_int, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.orc_contract.argtypes = [ip, C.c_int, C.c_int, ip, C.c_void_p, C.c_int, ip, C.c_void_p,
                                   C.c_int, ip, C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_int,
                                   C.c_int, C.c_int]
        L.orc_contract_blas.argtypes = [ip, C.c_int, C.c_int, ip, C.c_void_p, C.c_int, ip, C.c_void_p,
                                        C.c_int, ip, C.c_void_p, C.c_double, C.c_double, C.c_int,
                                        C.c_int]
        L.orc_blas_load.argtypes = [C.c_char_p]
        _lib = L
    return _lib


def _iarr(vals):
    vals = list(vals)
    return (C.c_int * max(1, len(vals)))(*vals)


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


def nthreads_default() -> int:
    return len(os.sched_getaffinity(0))


# ---------------------------------------------------------------- patterns --
class PatternError(ValueError):
    def __init__(self, code):
        super().__init__(f"pattern parse error {code}")
        self.code = code


def parse_pattern(pattern: str):
    """get_contr_pattern_dig: returns (cptrn list, drank, lrank, rrank, conj_bits).

    For a unary pattern (copy/add) rrank is -1 and cptrn has lrank entries."""
    cp = (C.c_int * 256)()
    d, l, r, cj = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    err = lib().orc_parse_pattern(pattern.encode(), cp, C.byref(d), C.byref(l), C.byref(r), C.byref(cj))
    if err:
        raise PatternError(err)
    n = l.value + max(r.value, 0)
    return list(cp[:n]), d.value, l.value, r.value, cj.value


def contr_permutations(cptrn, lrank, rrank, conj_bits=0, gemm_tl=1, gemm_tr=0):
    """get_contr_permutations: returns (dprm, lprm, rprm, ncd, nlu, nru), 1-based lists."""
    dp, lp, rp = (C.c_int * 64)(), (C.c_int * 64)(), (C.c_int * 64)()
    ncd, nlu, nru = C.c_int(), C.c_int(), C.c_int()
    err = lib().orc_contr_permutations(gemm_tl, gemm_tr, lrank, rrank, _iarr(cptrn), conj_bits,
                                       dp, lp, rp, C.byref(ncd), C.byref(nlu), C.byref(nru))
    if err:
        raise PatternError(err)
    drank = nlu.value + nru.value
    return (list(dp[1:drank + 1]), list(lp[1:lrank + 1]), list(rp[1:rrank + 1]),
            ncd.value, nlu.value, nru.value)


# -------------------------------------------------------------- operations --
def _dtk(a: np.ndarray) -> int:
    return DTK_OF[a.dtype]


def permute(a: np.ndarray, dims, o2n, conj=False, nthreads=None) -> np.ndarray:
    """tensor_block_copy with an O2N permutation (1-based): out(y), y(o2n(i)) = x(i)."""
    dims = list(dims)
    out = np.empty(int(np.prod(dims, dtype=np.int64)), dtype=a.dtype)
    err = lib().orc_permute(_dtk(a), len(dims), _iarr(dims), _iarr(o2n), _ptr(a), _ptr(out),
                            int(conj), nthreads or nthreads_default())
    assert err == 0
    return out


def permute_blocked(a: np.ndarray, dims, o2n, nthreads=None) -> np.ndarray:
    """Cache-blocked OpenMP permutation (the timed CPU baseline)."""
    dims = list(dims)
    out = np.empty(int(np.prod(dims, dtype=np.int64)), dtype=a.dtype)
    err = lib().orc_permute_blocked(_dtk(a), len(dims), _iarr(dims), _iarr(o2n), _ptr(a), _ptr(out),
                                    nthreads or nthreads_default())
    assert err == 0
    return out


def permuted_dims(dims, o2n):
    out = [0] * len(dims)
    for i, p in enumerate(o2n):
        out[p - 1] = dims[i]
    return out


def add(d: np.ndarray, l: np.ndarray, scale=1.0, conj_bits=0, accumulative=True, nthreads=None):
    """tensor_block_add in place on d: d = d + l*scale (or d = l*scale)."""
    s = complex(scale)
    err = lib().orc_add(_dtk(d), d.size, _ptr(d), _ptr(l), s.real, s.imag, conj_bits,
                        int(accumulative), nthreads or nthreads_default())
    assert err == 0
    return d


def tensor_add(cptrn, d: np.ndarray, l: np.ndarray, ldims, scale=1.0, conj_bits=0, nthreads=None):
    """cpu_tensor_block_add: permute-then-add, in place on d."""
    s = complex(scale)
    err = lib().orc_tensor_add(_iarr(cptrn), _dtk(d), len(ldims), _iarr(ldims), _ptr(d), _ptr(l),
                               s.real, s.imag, conj_bits, nthreads or nthreads_default())
    assert err == 0
    return d


def scale(d: np.ndarray, s):
    s = complex(s)
    assert lib().orc_scale(_dtk(d), d.size, _ptr(d), s.real, s.imag) == 0
    return d


def init(d: np.ndarray, v):
    v = complex(v)
    assert lib().orc_init(_dtk(d), d.size, _ptr(d), v.real, v.imag) == 0
    return d


def norm1(d: np.ndarray) -> float:
    return lib().orc_norm(_dtk(d), d.size, _ptr(d), 1)


def norm2sq(d: np.ndarray) -> float:
    return lib().orc_norm(_dtk(d), d.size, _ptr(d), 2)


def contract(cptrn, d, ddims, l, ldims, r, rdims, alpha=1.0, conj_bits=0, accumulative=True,
             mode=0, nthreads=None):
    """tensor_block_contract in place on d.  mode 0: TTGT in the data type;
    mode 1: double-double accumulation rounded once (the FP64 error oracle)."""
    a = complex(alpha)
    err = lib().orc_contract(_iarr(cptrn), _dtk(d), len(ddims), _iarr(ddims), _ptr(d),
                             len(ldims), _iarr(ldims), _ptr(l), len(rdims), _iarr(rdims), _ptr(r),
                             a.real, a.imag, conj_bits, int(accumulative), mode,
                             nthreads or nthreads_default())
    if err:
        raise PatternError(err)
    return d


def dd_dot_batch(l: np.ndarray, r: np.ndarray, nthreads=None) -> np.ndarray:
    """Row-wise dot products of two (n, K) float64 or complex128 arrays with
    double-double accumulation, rounded once (the FP64 error oracle for
    sampled elements of large contractions)."""
    l = np.ascontiguousarray(l)
    r = np.ascontiguousarray(r)
    assert l.shape == r.shape and l.ndim == 2 and l.dtype == r.dtype
    out = np.empty(l.shape[0], dtype=l.dtype)
    err = lib().orc_dd_dot_batch(_dtk(l), l.shape[0], l.shape[1], _ptr(l), _ptr(r), _ptr(out),
                                 nthreads or nthreads_default())
    if err:
        raise ValueError(f"orc_dd_dot_batch error {err}")
    return out


def blas_available() -> bool:
    for p in OPENBLAS_CANDIDATES:
        if os.path.exists(p) and lib().orc_blas_load(p.encode()) == 0:
            return True
    return False


def contract_blas(cptrn, d, ddims, l, ldims, r, rdims, alpha=1.0, accumulative=True, nthreads=None):
    """The reference's OpenMP+BLAS CPU contraction path (R4/R8), in place on d."""
    a = complex(alpha)
    err = lib().orc_contract_blas(_iarr(cptrn), _dtk(d), len(ddims), _iarr(ddims), _ptr(d),
                                  len(ldims), _iarr(ldims), _ptr(l), len(rdims), _iarr(rdims), _ptr(r),
                                  a.real, a.imag, int(accumulative), nthreads or nthreads_default())
    if err:
        raise RuntimeError(f"orc_contract_blas error {err}")
    return d


# ------------------------------------------------------------ input data --
def splitmix64_uniform(n: int, seed: int, lo=-1.0, hi=1.0) -> np.ndarray:
    """Seeded U[lo,hi) doubles: splitmix64 stream -> 53-bit mantissa fraction.
    The same generator is implemented on the GPU by exatensor_b200 (tb_fill_uniform)."""
    idx = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (np.uint64(seed) + (idx + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return lo + (hi - lo) * u


def fill_uniform(n: int, seed: int, lo=-1.0, hi=1.0, nthreads=None) -> np.ndarray:
    """splitmix64_uniform computed by the C oracle on all host threads (the
    same bits; for the large CPU-baseline operands)."""
    out = np.empty(n, dtype=np.float64)
    lib().orc_fill_uniform(n, seed, lo, hi, _ptr(out), nthreads or nthreads_default())
    return out


def rel_frobenius(x: np.ndarray, ref: np.ndarray) -> float:
    num = np.linalg.norm((x.astype(np.complex128) - ref.astype(np.complex128)).ravel())
    den = np.linalg.norm(ref.astype(np.complex128).ravel())
    return float(num / den) if den > 0 else float(num)


def max_abs_err(x: np.ndarray, ref: np.ndarray) -> float:
    return float(np.max(np.abs(x.astype(np.complex128) - ref.astype(np.complex128)))) if x.size else 0.0
