"""GPU parity against the REFERENCE'S OWN device kernels: this library's
copies, adds and contractions compared with TAL-SH's NV-TAL path
(TALSH/tensor_algebra_gpu_nvidia.cu: gpu_tensor_block_copy :4806,
gpu_tensor_block_add :5203, gpu_tensor_block_contract_dlf :5847), compiled
from the reference's sources by `make -C oracle ref` into
oracle/_ref/libnvtal_ref.so and driven through the harness oracle/ref_nvtal.cpp
(as the reference's NV-TAL test, TALSH/test.cpp:1016-1110, drives it).

  * copies (every data kind, all 24 rank-4 permutations, random ranks 1-6,
    conjugation) must be bit-identical to the reference kernels' results --
    except that NV-TAL's copy never conjugates (it computes the flag at :4887
    and passes it to no kernel), so conjugating copies are compared with its
    result conjugated, which is what its CPU path and its add compute;
  * adds (scale 1, 0.37 and complex, conjugation) give the CPU path's bits
    (two roundings), agree with NV-TAL's add kernel bit for bit at scale 1
    and otherwise within the product's rounding (2 eps (|d| + |l alpha|)):
    nvcc contracts its d + l*alpha into one FMA;
  * contractions (TTGT and the tensor-core method) agree with the reference's
    TTGT path (its permutation kernels and cuBLAS GEMMs, the reference's default
    build) within the relative Frobenius bounds of the methods
    (1e-13 / 1e-12 for R8/C8, 2e-5 / 1e-4 for R4/C4): the summation orders
    differ, so the bits do not;
  * the seeded 40^4 single-block contraction (seed 0, alpha 0.5, D = 0) agrees
    with the reference's within 1e-13 (TTGT) and 1e-12 (tensor cores).

The reference's NV-TAL initialisation reserves 90% of the free GPU memory for
its argument buffers, so the comparisons run in a child process of their own.
Full contractions to a scalar are not run through the reference: its dot
product kernel synchronises thread blocks with an unbounded spin lock
(gpu_array_dot_product__, :531-557)."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libnvtal_ref.so")


def child():
    import ctypes as C
    import itertools
    import random

    import numpy as np
    import torch

    sys.path.insert(0, ROOT)
    import exatensor_b200 as XB
    import oracle as O
    from tests.test_gpu_permute import rand_host

    XB.device_init(0)
    torch.zeros(1, device="cuda")
    R = C.CDLL(REF_LIB)
    ip, vp = C.POINTER(C.c_int), C.c_void_p
    R.ref_init.argtypes = [C.c_int]
    R.ref_copy.argtypes = [C.c_int, C.c_int, ip, ip, vp, vp, C.c_int]
    R.ref_add.argtypes = [C.c_int, C.c_int, ip, ip, vp, vp, C.c_double, C.c_double, C.c_int]
    R.ref_contract.argtypes = [ip, C.c_int, C.c_int, ip, vp, C.c_int, ip, vp, C.c_int, ip, vp, C.c_double,
                               C.c_double, C.c_int, C.c_int]
    arr = lambda v: (C.c_int * max(1, len(v)))(*[int(x) for x in v])
    ptr = lambda a: C.c_void_p(a.ctypes.data)
    assert R.ref_init(0) == 0
    s = torch.cuda.current_stream().cuda_stream
    out = {"copy": 0, "copy_conj": 0, "copy_fail": [], "add": 0, "add_exact": 0, "add_ulp_max": 0, "add_fail": [],
           "contract": 0, "contract_fail": [], "c1": {}}

    def put(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()

    def ours_copy(x, dims, perm, conj):
        src, dst = put(x), torch.empty(x.nbytes, dtype=torch.uint8, device="cuda")
        XB.tensor_copy(O.DTK_OF[x.dtype], dims, perm, src.data_ptr(), dst.data_ptr(), conj, s)
        torch.cuda.synchronize()
        return dst.cpu().numpy().view(x.dtype)

    def ref_copy(x, dims, perm, conj):
        d = np.empty_like(x)
        rc = R.ref_copy(O.DTK_OF[x.dtype], len(dims), arr(dims), arr(perm), ptr(x), ptr(d), conj)
        assert rc == 0, ("ref_copy", rc)
        return d

    def check_copy(x, dims, perm, conj=0):
        a, b = ours_copy(x, dims, perm, conj), ref_copy(x, dims, perm, conj)
        if ((conj & 1) ^ ((conj >> 1) & 1)) and np.iscomplexobj(x):
            # NV-TAL's copy computes the left argument's conjugation flag
            # (tensor_algebra_gpu_nvidia.cu:4883-4887) but passes it to no
            # kernel (:5101-5142): its GPU copies never conjugate.  Its CPU
            # path (tensor_block_copy, tensor_algebra_cpu.F90:3151-3310) and
            # its add (:5726-5731) do, and so does this library: the bits are
            # compared with the reference's result conjugated.
            b = np.conj(b)
            out["copy_conj"] += 1
        out["copy"] += 1
        if not np.array_equal(a.view(np.uint8), b.view(np.uint8)):
            out["copy_fail"].append([str(x.dtype), dims, list(perm), conj])

    for dtk in (O.R4, O.R8, O.C4, O.C8):
        dims = [5, 7, 3, 6]
        x = rand_host(dtk, int(np.prod(dims)), 11)
        for perm in itertools.permutations([1, 2, 3, 4]):
            check_copy(x, dims, perm)
        rng = random.Random(7 + dtk)
        for case in range(20):
            rank = rng.randint(1, 6)
            dims = [rng.choice([1, 2, 3, 5, 8, 13, 31, 40]) for _ in range(rank)]
            while np.prod(dims) > 200000:
                dims[int(np.argmax(dims))] //= 2
            perm = list(range(1, rank + 1))
            rng.shuffle(perm)
            check_copy(rand_host(dtk, int(np.prod(dims)), case), dims, perm)
        if dtk in (O.C4, O.C8):
            x = rand_host(dtk, 9 * 4 * 11, 3)
            for conj in (1, 2, 3):
                check_copy(x, [9, 4, 11], [2, 3, 1], conj)
    # larger copies that take the tiled kernel's multi-chunk paths in both libraries
    for dtk, dims, perm in ((O.R8, [64, 48, 40, 32], (3, 1, 4, 2)), (O.R4, [90, 90, 30, 30], (2, 4, 1, 3)),
                            (O.C8, [40, 40, 40, 40], (4, 3, 2, 1))):
        check_copy(rand_host(dtk, int(np.prod(dims)), 5), dims, perm)

    def ulps(a, b):
        """Largest distance in units in the last place between same-kind arrays."""
        w = np.int32 if a.dtype in (np.float32, np.complex64) else np.int64
        x = a.view(w).astype(np.int64)
        y = b.view(w).astype(np.int64)
        return int(np.max(np.abs(x - y))) if x.size else 0

    def check_add(dtk, dims, perm, scale, conj):
        n = int(np.prod(dims))
        l, d0 = rand_host(dtk, n, 21), rand_host(dtk, n, 22)
        dd, ld = put(d0), put(l)
        XB.tensor_add(dtk, dims, perm, dd.data_ptr(), ld.data_ptr(), scale, conj, s)
        torch.cuda.synchronize()
        mine = dd.cpu().numpy().view(d0.dtype)
        theirs = d0.copy()
        sc = complex(scale)
        rc = R.ref_add(dtk, len(dims), arr(dims), arr(perm), ptr(theirs), ptr(l), sc.real, sc.imag, conj)
        assert rc == 0, ("ref_add", rc)
        out["add"] += 1
        # the CPU path's bits (d + l*scale rounded twice) are the target
        cpu = O.tensor_add(list(perm), d0.copy(), l, dims, scale, conj)
        if not np.array_equal(mine.view(np.uint8), cpu.view(np.uint8)):
            out["add_fail"].append(["cpu", dtk, dims, list(perm), str(scale), conj])
        if np.array_equal(mine.view(np.uint8), theirs.view(np.uint8)):
            out["add_exact"] += 1
        else:
            # NV-TAL's gpu_array_add__ (:443-526) is compiled with nvcc's default
            # -fmad=true, which contracts arr0 + arr1*alpha into one FMA (one
            # rounding); the CPU path rounds twice.  Where alpha = 1 the product
            # is exact and the two agree bit for bit; otherwise they differ by at
            # most the product's rounding, eps * |l * alpha| (plus the sum's).
            eps = 2.0 ** -23 if d0.dtype in (np.float32, np.complex64) else 2.0 ** -52
            lp = O.permute(l, dims, list(perm)).astype(np.complex128)
            bound = 2 * eps * (np.abs(d0.astype(np.complex128)) + np.abs(lp) * abs(complex(scale)))
            diff = np.abs(mine.astype(np.complex128) - theirs.astype(np.complex128))
            out["add_ulp_max"] = max(out["add_ulp_max"], ulps(mine, theirs))
            if complex(scale) == 1 or not np.all(diff <= bound):
                out["add_fail"].append(["gpu", dtk, dims, list(perm), str(scale), conj, float(np.max(diff / bound))])

    for dtk in (O.R4, O.R8, O.C4, O.C8):
        for perm in list(itertools.permutations([1, 2, 3, 4]))[::3]:
            for scale in ([1.0, 0.37] + ([-2.5 + 0.75j] if dtk in (O.C4, O.C8) else [])):
                check_add(dtk, [6, 5, 4, 7], perm, scale, 0)
        if dtk in (O.C4, O.C8):
            for conj in (2, 3):
                check_add(dtk, [6, 5, 4, 7], (2, 1, 4, 3), 0.5 - 0.25j, conj)

    def check_contract(pattern, ext, dtk, method, alpha, accumulative, seed=1):
        from tests.test_gpu_contract import shapes
        ddims, ldims, rdims = shapes(pattern, ext)
        vol = lambda q: int(np.prod(q)) if q else 1
        d, l, r = rand_host(dtk, vol(ddims), seed), rand_host(dtk, vol(ldims), seed + 1), rand_host(dtk, vol(rdims),
                                                                                                      seed + 2)
        cptrn, _, _, _, cj = O.parse_pattern(pattern)
        dd, ld, rd = put(d), put(l), put(r)
        XB.tensor_contract(cptrn, dtk, ddims, dd.data_ptr(), ldims, ld.data_ptr(), rdims, rd.data_ptr(), alpha,
                           cj, accumulative, XB.make_plan(method), s)
        torch.cuda.synchronize()
        mine = dd.cpu().numpy().view(d.dtype)
        st = XB.last_contract_stats()
        theirs = d.copy()
        a = complex(alpha)
        rc = R.ref_contract(arr(cptrn), dtk, len(ddims), arr(ddims), ptr(theirs), len(ldims), arr(ldims), ptr(l),
                            len(rdims), arr(rdims), ptr(r), a.real, a.imag, cj, int(accumulative))
        assert rc == 0, ("ref_contract", rc, pattern)
        tol = {(XB.METHOD_TTGT, O.R8): 1e-13, (XB.METHOD_TTGT, O.C8): 1e-13, (XB.METHOD_TTGT, O.R4): 2e-5,
               (XB.METHOD_TTGT, O.C4): 2e-5, (XB.METHOD_FUSED, O.R8): 1e-12, (XB.METHOD_FUSED, O.C8): 1e-12,
               (XB.METHOD_FUSED, O.R4): 1e-4, (XB.METHOD_FUSED, O.C4): 1e-4}[(st.method, dtk)]
        err = O.rel_frobenius(mine, theirs)
        out["contract"] += 1
        if not err <= tol:
            out["contract_fail"].append([pattern, dtk, st.method, err])
        return err

    cases = [("D(a,b,c,d)+=L(c,k,a,l)*R(l,d,k,b)", {"a": 12, "b": 11, "c": 13, "d": 10, "k": 9, "l": 14}),
             ("D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)", {"a": 16, "b": 16, "c": 16, "d": 16, "i": 8, "j": 8}),
             ("D(a,i,b,j)+=L(a,k,c,i)*R(c,b,k,j)", {"a": 16, "b": 16, "c": 16, "i": 8, "j": 8, "k": 8}),
             ("D(j,i)+=L(i,k)*R(j,k)", {"i": 300, "j": 200, "k": 128}),
             ("D(a,b,c)+=L(a,c)*R(b)", {"a": 20, "b": 30, "c": 10})]
    for dtk in (O.R8, O.R4, O.C8, O.C4):
        for pattern, ext in cases:
            for method in (XB.METHOD_TTGT, XB.METHOD_FUSED):
                if method == XB.METHOD_FUSED and "L(a,c)*R(b)" in pattern:
                    continue  # no contracted index: the tensor-core path does not apply
                check_contract(pattern, ext, dtk, method, 0.5, True)
                check_contract(pattern, ext, dtk, method, -1.25, False)
    for dtk in (O.C8, O.C4):
        for pattern in ("D(a,b)+=L+(k,a)*R(k,b)", "D(a,b)+=L(k,a)*R+(k,b)"):
            for method in (XB.METHOD_TTGT, XB.METHOD_FUSED):
                check_contract(pattern, {"a": 70, "b": 50, "k": 90}, dtk, method, 0.7 - 0.2j, True)

    # the seeded single-block 40^4 configuration (seed 0, L then R, alpha 0.5, D = 0)
    pat, dims, vol = "D(a,b,c,d)+=L(c,k,a,l)*R(l,d,k,b)", [40] * 4, 40 ** 4
    u = O.splitmix64_uniform(2 * vol, 0)
    L, Rr = u[:vol].copy(), u[vol:].copy()
    cptrn, *_ = O.parse_pattern(pat)
    theirs = np.zeros(vol)
    assert R.ref_contract(arr(cptrn), O.R8, 4, arr(dims), ptr(theirs), 4, arr(dims), ptr(L), 4, arr(dims), ptr(Rr),
                          0.5, 0.0, 0, 1) == 0
    for method in (XB.METHOD_TTGT, XB.METHOD_FUSED):
        dd, ld, rd = put(np.zeros(vol)), put(L), put(Rr)
        XB.tensor_contract(cptrn, O.R8, dims, dd.data_ptr(), dims, ld.data_ptr(), dims, rd.data_ptr(), 0.5, 0, True,
                           XB.make_plan(method), s)
        torch.cuda.synchronize()
        out["c1"][str(method)] = O.rel_frobenius(dd.cpu().numpy().view(np.float64), theirs)
    XB.device_check(s)
    print("RESULT " + json.dumps(out))


@pytest.mark.skipif(not os.path.exists(REF_LIB),
                    reason="oracle/_ref/libnvtal_ref.so not built (`make -C oracle ref` needs the reference sources)")
def test_against_reference_nvtal_kernels():
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "child"], capture_output=True, text=True,
                       timeout=900, cwd=ROOT)
    line = [x for x in r.stdout.splitlines() if x.startswith("RESULT ")]
    assert r.returncode == 0 and line, (r.returncode, r.stdout[-2000:], r.stderr[-3000:])
    res = json.loads(line[-1][7:])
    assert res["copy"] >= 180 and not res["copy_fail"], res["copy_fail"][:5]
    assert res["add"] >= 40 and not res["add_fail"], res["add_fail"][:5]
    assert res["contract"] >= 60 and not res["contract_fail"], res["contract_fail"][:5]
    assert res["c1"][str(1)] <= 1e-13 and res["c1"][str(2)] <= 1e-12, res["c1"]


if __name__ == "__main__" and len(sys.argv) > 1 and sys.argv[1] == "child":
    child()
