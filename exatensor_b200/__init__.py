"""exatensor_b200: TAL-SH's device tensor-algebra path, native on B200 (sm_100a).

The compute lives in ``libtalsh_b200.so`` (hand-written CUDA for sm_100a plus
the C++ ``talsh.h`` layer), built in-tree by ``exatensor_b200.build``.  This
module is a thin ctypes binding of its C ABI (``include/talsh_b200.h``) for
Python callers and the test-suite; device memory is passed as raw pointers
(e.g. ``torch.Tensor.data_ptr()``) and streams as ``cudaStream_t`` handles.

There is no Python or CPU fallback: if the library is missing or no B200 is
visible, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

R4, R8, C4, C8 = 4, 8, 14, 18
DATA_KINDS = (R4, R8, C4, C8)
ELEM_BYTES = {R4: 4, R8: 8, C4: 8, C8: 16}

TB_SUCCESS = 0
TB_ERR = {1: "invalid arguments", 2: "bad pattern", 3: "CUDA error", 4: "not implemented", 5: "device error",
          6: "out of memory", 7: "limit exceeded"}
METHOD_AUTO, METHOD_TTGT, METHOD_FUSED = 0, 1, 2

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtalsh_b200.so")
_lib = None


class TBError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{TB_ERR.get(code, 'error')} ({code}): {msg}")
        self.code = code


class Plan(C.Structure):
    """tb_plan_t: contraction plan (method, INT8 slices, N tile, split-BF16 terms, M tile)."""
    _fields_ = [("method", C.c_int), ("slices", C.c_int), ("tile_n", C.c_int), ("bf16_terms", C.c_int),
                ("tile_m", C.c_int), ("moduli", C.c_int), ("reserved", C.c_int * 2)]


class ContractStats(C.Structure):
    _fields_ = [("method", C.c_int), ("slices", C.c_int), ("passes", C.c_int), ("gemm_launches", C.c_int),
                ("m", C.c_longlong), ("n", C.c_longlong), ("k", C.c_longlong), ("flops", C.c_double),
                ("products", C.c_int), ("tile_n", C.c_int), ("tile_m", C.c_int), ("moduli", C.c_int),
                ("residue_bits", C.c_int)]


class BlockTask(C.Structure):
    """tb_block_task_t: one block contraction of a block-sparse list."""
    _fields_ = [("d", C.c_void_p), ("l", C.c_void_p), ("r", C.c_void_p), ("d_dims", C.c_int * 8),
                ("l_dims", C.c_int * 8), ("r_dims", C.c_int * 8)]


class BlockList(C.Structure):
    """tb_block_list_t: segment metadata and present blocks of a block-sparse tensor."""
    _fields_ = [("rank", C.c_int), ("nseg", C.POINTER(C.c_int)), ("seg_ext", C.POINTER(C.c_int)),
                ("nblocks", C.c_int), ("keys", C.POINTER(C.c_int)), ("bodies", C.POINTER(C.c_void_p))]


class BatchStats(C.Structure):
    _fields_ = [("tasks", C.c_longlong), ("grouped_flushes", C.c_int), ("loop_flushes", C.c_int),
                ("plans_built", C.c_int), ("plan_reuses", C.c_int), ("autotunes", C.c_int),
                ("cached_plans", C.c_int)]


class BscInfo(C.Structure):
    _fields_ = [("tasks", C.c_int), ("left_blocks", C.c_int), ("right_blocks", C.c_int), ("out_blocks", C.c_int),
                ("work_items", C.c_int), ("slices", C.c_int), ("tile_n", C.c_int), ("flops", C.c_double),
                ("tune_ms", C.c_float * 4)]


def lib() -> C.CDLL:
    """Loads libtalsh_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m exatensor_b200.build`")
    L = C.CDLL(LIB_PATH)
    ip, vp, i64 = C.POINTER(C.c_int), C.c_void_p, C.c_int64
    L.tb_last_error.restype = C.c_char_p
    L.tb_launch_count.restype = C.c_longlong
    L.tb_timing_enable.argtypes = [C.c_int]
    L.tb_timing_read.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_int)]
    L.tb_device_init.argtypes = [C.c_int]
    L.tb_device_check.argtypes = [vp]
    L.tb_data_kind_size.argtypes = [C.c_int]
    L.tb_parse_pattern.argtypes = [C.c_char_p, ip, ip, ip, ip, ip]
    L.tb_tensor_copy.argtypes = [C.c_int, C.c_int, ip, ip, vp, vp, C.c_int, vp]
    L.tb_tensor_copy_scatter.argtypes = [C.c_int, C.c_int, ip, ip, vp, vp, C.c_int, vp]
    L.tb_tensor_add.argtypes = [C.c_int, C.c_int, ip, ip, vp, vp, C.c_double, C.c_double, C.c_int, vp]
    L.tb_tensor_init.argtypes = [C.c_int, C.c_size_t, vp, C.c_double, C.c_double, vp]
    L.tb_tensor_scale.argtypes = [C.c_int, C.c_size_t, vp, C.c_double, C.c_double, vp]
    L.tb_tensor_norm.argtypes = [C.c_int, C.c_size_t, vp, C.c_int, C.POINTER(C.c_double), vp]
    L.tb_tensor_contract.argtypes = [ip, C.c_int, C.c_int, ip, vp, C.c_int, ip, vp, C.c_int, ip, vp, C.c_double,
                                     C.c_double, C.c_int, C.c_int, C.POINTER(Plan), vp]
    L.tb_tensor_contract_str.argtypes = [C.c_char_p, C.c_int, C.c_int, ip, vp, C.c_int, ip, vp, C.c_int, ip, vp,
                                         C.c_double, C.c_double, C.c_int, C.POINTER(Plan), vp]
    L.tb_tensor_contract_noalloc.argtypes = [ip, C.c_int, C.c_int, ip, vp, C.c_int, ip, vp, C.c_int, ip, vp,
                                             C.c_double, C.c_double, C.c_int, C.c_int, vp]
    L.tb_bsc_plan_create.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(BlockTask), C.c_double, C.c_double,
                                     C.c_int, C.POINTER(Plan), C.POINTER(C.c_void_p), vp]
    L.tb_bsc_execute.argtypes = [vp, vp]
    L.tb_bsc_execute_stream.argtypes = [vp, vp]
    L.tb_bsc_autotune.argtypes = [vp, vp]
    L.tb_bsc_plan_info.argtypes = [vp, C.POINTER(BscInfo)]
    L.tb_bsc_plan_destroy.argtypes = [vp]
    bl = C.POINTER(BlockList)
    L.tb_bsc_tasks_from_blocks.argtypes = [C.c_char_p, bl, bl, bl, C.c_int, C.POINTER(BlockTask), ip]
    L.tb_batch_create.argtypes = [C.c_char_p, C.c_int, C.c_double, C.c_double, C.c_int, C.POINTER(Plan),
                                  C.POINTER(C.c_void_p)]
    L.tb_batch_add.argtypes = [vp, C.c_int, C.POINTER(BlockTask)]
    L.tb_batch_pending.argtypes = [vp]
    L.tb_batch_flush.argtypes = [vp, vp]
    L.tb_batch_get_stats.argtypes = [vp, C.POINTER(BatchStats)]
    L.tb_batch_destroy.argtypes = [vp]
    fp = C.POINTER(C.c_float)
    L.tb_contract_descriptor.argtypes = [ip, C.c_int, C.c_int, ip, C.c_int, ip, C.c_int, ip, fp]
    L.tb_mlp_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]
    L.tb_mlp_destroy.argtypes = [vp]
    L.tb_mlp_num_params.argtypes = [vp]
    L.tb_mlp_num_params.restype = C.c_longlong
    L.tb_mlp_get_params.argtypes = [vp, fp, C.c_int]
    L.tb_mlp_set_params.argtypes = [vp, fp]
    L.tb_mlp_forward.argtypes = [vp, vp, C.c_int, vp, vp]
    L.tb_mlp_backward.argtypes = [vp, vp, vp, C.c_int, fp, vp]
    L.tb_mlp_adam_step.argtypes = [vp, C.c_float, C.c_float, C.c_float, C.c_float, vp]
    L.tb_selector_install.argtypes = [C.c_int, fp, fp, fp, C.c_float, C.c_int]
    L.tb_selector_choose.argtypes = [fp, fp]
    L.tb_selector_time.argtypes = [fp, C.c_int, C.POINTER(C.c_double)]
    L.tb_fill_uniform.argtypes = [C.c_int, C.c_size_t, vp, C.c_uint64, C.c_double, C.c_double, vp]
    L.tb_last_contract_stats.argtypes = [C.POINTER(ContractStats)]
    L.tb_peak_measure.argtypes = [C.c_int, C.c_longlong, C.POINTER(C.c_double), C.POINTER(C.c_double), vp]
    _lib = L
    return L


def _check(code: int):
    if code != TB_SUCCESS:
        raise TBError(code, lib().tb_last_error().decode(errors="replace"))


def iarr(vals) -> C.Array:
    vals = [int(v) for v in vals]
    return (C.c_int * max(1, len(vals)))(*vals)


def _stream(stream):
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return C.c_void_p(stream.cuda_stream)
    return C.c_void_p(int(stream))


def device_init(gpu: int = 0):
    _check(lib().tb_device_init(gpu))


def device_check(stream=None):
    _check(lib().tb_device_check(_stream(stream)))


def parse_pattern(pattern: str):
    """Symbolic -> digital pattern: (cptrn, drank, lrank, rrank, conj_bits); rrank=-1 for unary."""
    cp = (C.c_int * 112)()
    d, l, r, cj = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    _check(lib().tb_parse_pattern(pattern.encode(), cp, C.byref(d), C.byref(l), C.byref(r), C.byref(cj)))
    n = l.value + max(r.value, 0)
    return list(cp[:n]), d.value, l.value, r.value, cj.value


def tensor_copy(dtk, dims, cptrn, src_ptr, dst_ptr, conj_bits=0, stream=None, scatter=False):
    f = lib().tb_tensor_copy_scatter if scatter else lib().tb_tensor_copy
    _check(f(dtk, len(dims), iarr(dims), iarr(cptrn), C.c_void_p(src_ptr), C.c_void_p(dst_ptr), conj_bits,
             _stream(stream)))


def tensor_add(dtk, ldims, cptrn, d_ptr, l_ptr, scale=1.0, conj_bits=0, stream=None):
    s = complex(scale)
    _check(lib().tb_tensor_add(dtk, len(ldims), iarr(ldims), iarr(cptrn), C.c_void_p(d_ptr), C.c_void_p(l_ptr),
                               s.real, s.imag, conj_bits, _stream(stream)))


def tensor_init(dtk, volume, d_ptr, value=0.0, stream=None):
    v = complex(value)
    _check(lib().tb_tensor_init(dtk, volume, C.c_void_p(d_ptr), v.real, v.imag, _stream(stream)))


def tensor_scale(dtk, volume, d_ptr, scale, stream=None):
    s = complex(scale)
    _check(lib().tb_tensor_scale(dtk, volume, C.c_void_p(d_ptr), s.real, s.imag, _stream(stream)))


def tensor_norm(dtk, volume, d_ptr, which=1, stream=None) -> float:
    out = C.c_double()
    _check(lib().tb_tensor_norm(dtk, volume, C.c_void_p(d_ptr), which, C.byref(out), _stream(stream)))
    return out.value


def fill_uniform(dtk, volume, d_ptr, seed, lo=-1.0, hi=1.0, stream=None):
    _check(lib().tb_fill_uniform(dtk, volume, C.c_void_p(d_ptr), seed, lo, hi, _stream(stream)))


def make_plan(method=METHOD_AUTO, slices=0, tile_n=0, bf16_terms=0, tile_m=0, moduli=0) -> Plan:
    """moduli (R8/C8 on the tensor cores): 0 = modular residues where possible,
    8..15 = that many moduli, -1 = INT8 slices; slices > 0 also selects slices."""
    p = Plan()
    p.method, p.slices, p.tile_n, p.bf16_terms, p.tile_m = method, slices, tile_n, bf16_terms, tile_m
    p.moduli = moduli
    return p


def tensor_contract(pattern_or_cptrn, dtk, ddims, d_ptr, ldims, l_ptr, rdims, r_ptr, alpha=1.0, conj_bits=0,
                    accumulative=True, plan: Plan | None = None, stream=None):
    """D = beta*D + alpha*op(L)*op(R); pattern may be symbolic (str) or digital (list)."""
    a = complex(alpha)
    pp = C.byref(plan) if plan is not None else None
    if isinstance(pattern_or_cptrn, str):
        _check(lib().tb_tensor_contract_str(pattern_or_cptrn.encode(), dtk, len(ddims), iarr(ddims),
                                            C.c_void_p(d_ptr), len(ldims), iarr(ldims), C.c_void_p(l_ptr),
                                            len(rdims), iarr(rdims), C.c_void_p(r_ptr), a.real, a.imag,
                                            int(accumulative), pp, _stream(stream)))
    else:
        _check(lib().tb_tensor_contract(iarr(pattern_or_cptrn), dtk, len(ddims), iarr(ddims), C.c_void_p(d_ptr),
                                        len(ldims), iarr(ldims), C.c_void_p(l_ptr), len(rdims), iarr(rdims),
                                        C.c_void_p(r_ptr), a.real, a.imag, conj_bits, int(accumulative), pp,
                                        _stream(stream)))


def _task_array(tasks):
    tasks = list(tasks)
    arr = (BlockTask * max(1, len(tasks)))()
    for t, (dp, dd, lp, ld, rp, rd) in zip(arr, tasks):
        t.d, t.l, t.r = dp, lp, rp
        for k, v in enumerate(dd):
            t.d_dims[k] = v
        for k, v in enumerate(ld):
            t.l_dims[k] = v
        for k, v in enumerate(rd):
            t.r_dims[k] = v
    return arr, len(tasks)


def _block_list(segments, keys, bodies):
    """A BlockList over Python data; returns (struct, keepalive)."""
    rank = len(segments)
    nseg = iarr([len(s) for s in segments])
    ext = iarr([e for s in segments for e in s])
    flat = iarr([x for k in keys for x in k])
    bod = (C.c_void_p * max(1, len(bodies)))(*[int(b) for b in bodies])
    bl = BlockList(rank, nseg, ext, len(keys), flat, bod)
    return bl, (nseg, ext, flat, bod)


def bsc_tasks_from_blocks(pattern, d, l, r):
    """Block tasks of a block-sparse contraction from segment metadata (see
    tb_bsc_tasks_from_blocks).  d, l, r: (segments, keys, bodies) with
    segments[k] the extents of index k's segments, keys the present blocks'
    segment numbers and bodies their device addresses.  Returns a list of
    (d_ptr, d_dims, l_ptr, l_dims, r_ptr, r_dims)."""
    (bd, kd), (bl_, kl), (br, kr) = _block_list(*d), _block_list(*l), _block_list(*r)
    n = C.c_int()
    _check(lib().tb_bsc_tasks_from_blocks(pattern.encode(), C.byref(bd), C.byref(bl_), C.byref(br), 0, None,
                                          C.byref(n)))
    arr = (BlockTask * max(1, n.value))()
    _check(lib().tb_bsc_tasks_from_blocks(pattern.encode(), C.byref(bd), C.byref(bl_), C.byref(br), n.value, arr,
                                          C.byref(n)))
    dr, lr, rr = len(d[0]), len(l[0]), len(r[0])
    return [(t.d, list(t.d_dims[:dr]), t.l, list(t.l_dims[:lr]), t.r, list(t.r_dims[:rr])) for t in arr[:n.value]]


class Batch:
    """Caller-side batch of block contractions (tb_batch_*): add tasks one by
    one or in groups, flush them as one grouped launch."""

    def __init__(self, pattern, dtk, alpha=1.0, accumulative=True, plan: Plan | None = None):
        a = complex(alpha)
        h = C.c_void_p()
        _check(lib().tb_batch_create(pattern.encode(), dtk, a.real, a.imag, int(accumulative),
                                     C.byref(plan) if plan is not None else None, C.byref(h)))
        self._h = h

    def add(self, tasks):
        arr, n = _task_array(tasks)
        _check(lib().tb_batch_add(self._h, n, arr))

    def pending(self) -> int:
        return lib().tb_batch_pending(self._h)

    def flush(self, stream=None):
        _check(lib().tb_batch_flush(self._h, _stream(stream)))

    def stats(self) -> BatchStats:
        st = BatchStats()
        _check(lib().tb_batch_get_stats(self._h, C.byref(st)))
        return st

    def close(self):
        if self._h:
            lib().tb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BlockSparsePlan:
    """A block-sparse contraction (list of block tasks under one pattern) run as
    one grouped tensor-core launch; see tb_bsc_plan_create.

    tasks: iterable of (d_ptr, d_dims, l_ptr, l_dims, r_ptr, r_dims)."""

    def __init__(self, pattern, dtk, tasks, alpha=1.0, accumulative=True, plan: Plan | None = None, stream=None):
        arr, n = _task_array(tasks)
        a = complex(alpha)
        h = C.c_void_p()
        _check(lib().tb_bsc_plan_create(pattern.encode(), dtk, n, arr, a.real, a.imag, int(accumulative),
                                        C.byref(plan) if plan is not None else None, C.byref(h), _stream(stream)))
        self._h = h

    def execute(self, stream=None, graph=True):
        f = lib().tb_bsc_execute if graph else lib().tb_bsc_execute_stream
        _check(f(self._h, _stream(stream)))

    def autotune(self, stream=None):
        _check(lib().tb_bsc_autotune(self._h, _stream(stream)))

    def info(self) -> BscInfo:
        inf = BscInfo()
        _check(lib().tb_bsc_plan_info(self._h, C.byref(inf)))
        return inf

    def close(self):
        if self._h:
            lib().tb_bsc_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


DESC_FEATURES, SELECT_PLANS = 16, 5


def contract_descriptor(pattern, dtk, ddims, ldims, rdims):
    """Feature vector of a contraction (host only; see tb_contract_descriptor)."""
    import numpy as np
    cptrn, dr, lr, rr, _ = parse_pattern(pattern)
    f = (C.c_float * DESC_FEATURES)()
    _check(lib().tb_contract_descriptor(iarr(cptrn), dtk, len(ddims), iarr(ddims), len(ldims), iarr(ldims),
                                        len(rdims), iarr(rdims), f))
    return np.array(f[:], dtype=np.float32)


def _fptr(a):
    import numpy as np
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


class MLP:
    """The selector network on the GPU (tb_mlp_*): in -> hidden -> hidden -> out."""

    def __init__(self, n_in, n_hidden, n_out, max_batch=256, seed=1):
        h = C.c_void_p()
        _check(lib().tb_mlp_create(n_in, n_hidden, n_out, max_batch, seed, C.byref(h)))
        self._h, self.n_in, self.n_hidden, self.n_out, self.max_batch = h, n_in, n_hidden, n_out, max_batch
        self.n_params = int(lib().tb_mlp_num_params(h))

    def params(self, grads=False):
        import numpy as np
        out = np.empty(self.n_params, dtype=np.float32)
        _check(lib().tb_mlp_get_params(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), int(grads)))
        return out

    def set_params(self, p):
        a, ptr = _fptr(p)
        _check(lib().tb_mlp_set_params(self._h, ptr))

    def forward(self, x_dev_ptr, batch, y_dev_ptr, stream=None):
        _check(lib().tb_mlp_forward(self._h, C.c_void_p(x_dev_ptr), batch, C.c_void_p(y_dev_ptr), _stream(stream)))

    def backward(self, x_dev_ptr, t_dev_ptr, batch, stream=None, want_loss=True):
        loss = C.c_float()
        _check(lib().tb_mlp_backward(self._h, C.c_void_p(x_dev_ptr), C.c_void_p(t_dev_ptr), batch,
                                     C.byref(loss) if want_loss else None, _stream(stream)))
        return loss.value

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        _check(lib().tb_mlp_adam_step(self._h, lr, beta1, beta2, eps, _stream(stream)))

    def close(self):
        if self._h:
            lib().tb_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def selector_install(n_hidden, params, mean, scale, margin=0.0, autotune=False):
    """Installs a trained selector for METHOD_AUTO (params None removes it)."""
    if params is None:
        _check(lib().tb_selector_install(0, None, None, None, 0.0, 0))
        return
    _p, pp = _fptr(params)
    _m, mp = _fptr(mean)
    _s, sp = _fptr(scale)
    _check(lib().tb_selector_install(n_hidden, pp, mp, sp, float(margin), int(autotune)))


def selector_choose(features):
    """(plan index, predicted log-runtimes) for a descriptor, or (-1, None)."""
    import numpy as np
    _f, fp = _fptr(features)
    y = (C.c_float * SELECT_PLANS)()
    idx = lib().tb_selector_choose(fp, y)
    return idx, (np.array(y[:]) if idx >= 0 else None)


def selector_time(features, iters=10000) -> float:
    """Microseconds per selection (host inference timed inside the library)."""
    _f, fp = _fptr(features)
    us = C.c_double()
    if lib().tb_selector_time(fp, int(iters), C.byref(us)) != 0:
        raise TBError(-1, "no selector installed")
    return us.value


NOALLOC_ARENA_BYTES = 64 << 20  # TB_NOALLOC_ARENA_BYTES


def tensor_contract_noalloc(pattern_or_cptrn, dtk, ddims, d_ptr, ldims, l_ptr, rdims, r_ptr, alpha=1.0,
                            conj_bits=0, accumulative=True, stream=None):
    """Plain (TTGT) contraction that allocates no device memory: its scratch is
    a fixed static array of NOALLOC_ARENA_BYTES per device, so larger requests
    raise TBError (TB_ERR_LIMIT).  Same arguments as tensor_contract without a
    plan; calls that overlap on the GPU share the array and race."""
    a = complex(alpha)
    if isinstance(pattern_or_cptrn, str):
        cptrn, dr, lr, rr, conj_bits = parse_pattern(pattern_or_cptrn)
        if (dr, lr, rr) != (len(ddims), len(ldims), len(rdims)):
            raise TBError(1, "pattern ranks do not match the tensors")
    else:
        cptrn = pattern_or_cptrn
    _check(lib().tb_tensor_contract_noalloc(iarr(cptrn), dtk, len(ddims), iarr(ddims), C.c_void_p(d_ptr),
                                            len(ldims), iarr(ldims), C.c_void_p(l_ptr), len(rdims), iarr(rdims),
                                            C.c_void_p(r_ptr), a.real, a.imag, conj_bits, int(accumulative),
                                            _stream(stream)))


def launch_count() -> int:
    return lib().tb_launch_count()


def timing_enable(on: bool = True):
    lib().tb_timing_enable(int(on))


def timing_read():
    """(summed milliseconds, launches) of the timed GEMM kernels since the last read."""
    ms, n = C.c_double(), C.c_int()
    lib().tb_timing_read(C.byref(ms), C.byref(n))
    return ms.value, n.value


def last_contract_stats() -> ContractStats:
    st = ContractStats()
    _check(lib().tb_last_contract_stats(C.byref(st)))
    return st


PEAK_I8, PEAK_BF16, PEAK_F64 = 1, 2, 3


def peak_measure(kind, iters, stream=None):
    """(operations per second, milliseconds) of a tensor-core throughput probe
    (PEAK_I8, PEAK_BF16 or PEAK_F64) with operands resident on chip; see
    tb_peak_measure in include/talsh_b200.h.  Synchronizes the stream."""
    rate, ms = C.c_double(), C.c_double()
    _check(lib().tb_peak_measure(int(kind), int(iters), C.byref(rate), C.byref(ms), _stream(stream)))
    return rate.value, ms.value
