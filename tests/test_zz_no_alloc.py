"""GPU checks of tb_tensor_contract_noalloc: the plain (TTGT) contraction for
callers that may not allocate device memory while they run, whose scratch is a
fixed static device array instead of an allocation.

The file name makes pytest collect it last, so a run that stops at the first
failure has run every other test before it; it also passes on its own.  Each
case runs the existing entry point (tb_tensor_contract, method TTGT) once and
the no-alloc entry point twice in a row on the same inputs.  Both entry points
run the same kernels in the same order, so the three results must agree bit
for bit, and lie within the contraction tests' tolerance of the FP64
double-double oracle.
"""
import numpy as np
import pytest

import exatensor_b200 as XB
import oracle as O
from tests.test_gpu_contract import oracle_dd, shapes
from tests.test_gpu_permute import rand_host

pytestmark = pytest.mark.gpu
TOL = {O.R8: 1e-13, O.C8: 1e-13, O.R4: 2e-5, O.C4: 2e-5}   # as the TTGT contraction tests

CASES = [
    ("D(a,b,c,d)+=L(c,k,a,l)*R(l,d,k,b)", {"a": 12, "b": 11, "c": 13, "d": 10, "k": 9, "l": 14}, O.R8),
    ("D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)", {"a": 16, "b": 16, "c": 16, "d": 16, "i": 8, "j": 8}, O.R4),
    ("D(a,i,b,j)+=L+(a,k,c,i)*R(c,b,k,j)", {"a": 16, "b": 12, "c": 10, "i": 8, "j": 6, "k": 7}, O.C8),
    ("D(i,j)+=L(k,i)*R(k,j)", {"i": 300, "j": 200, "k": 128}, O.C4),   # matrix-shaped: no permutations
    ("D()+=L(a,b,c)*R(c,a,b)", {"a": 40, "b": 30, "c": 20}, O.R8),      # full contraction: dot partials
]


def _inputs(pattern, ext, dtk, seed):
    ddims, ldims, rdims = shapes(pattern, ext)
    vol = lambda s: int(np.prod(s)) if s else 1
    return (ddims, ldims, rdims, rand_host(dtk, vol(ddims), seed), rand_host(dtk, vol(ldims), seed + 1),
            rand_host(dtk, vol(rdims), seed + 2))


def _run(xt, dev, fn, pattern, dtk, ddims, d, ldims, l, rdims, r, alpha, **kw):
    dd, ld, rd = dev.put(d), dev.put(l), dev.put(r)
    fn(pattern, dtk, ddims, dd.data_ptr(), ldims, ld.data_ptr(), rdims, rd.data_ptr(), alpha,
       accumulative=True, stream=dev.stream(), **kw)
    out = dev.get(dd, d.dtype, d.size)
    xt.device_check(dev.stream())
    return out


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"dtk{c[2]}-{c[0]}")
def test_noalloc_matches_contract_twice(xt, dev, case):
    pattern, ext, dtk = case
    ddims, ldims, rdims, d, l, r = _inputs(pattern, ext, dtk, 7)
    alpha = 0.75 - (0.25j if dtk in (O.C4, O.C8) else 0)
    ref = _run(xt, dev, xt.tensor_contract, pattern, dtk, ddims, d, ldims, l, rdims, r, alpha,
               plan=xt.make_plan(XB.METHOD_TTGT))
    first = _run(xt, dev, xt.tensor_contract_noalloc, pattern, dtk, ddims, d, ldims, l, rdims, r, alpha)
    assert xt.last_contract_stats().method == XB.METHOD_TTGT
    second = _run(xt, dev, xt.tensor_contract_noalloc, pattern, dtk, ddims, d, ldims, l, rdims, r, alpha)
    assert np.array_equal(first.view(np.uint8), ref.view(np.uint8))
    assert np.array_equal(second.view(np.uint8), ref.view(np.uint8))
    exact = oracle_dd(pattern, d, ddims, l, ldims, r, rdims, alpha, True)
    assert O.rel_frobenius(first, exact) <= TOL[dtk]


def test_noalloc_back_to_back_different_shapes(xt, dev):
    """Consecutive calls with different shapes: the second must not depend on
    what the first left in the shared scratch array."""
    for pattern, ext, dtk in (CASES[0], CASES[2], CASES[0]):
        ddims, ldims, rdims, d, l, r = _inputs(pattern, ext, dtk, 11)
        ref = _run(xt, dev, xt.tensor_contract, pattern, dtk, ddims, d, ldims, l, rdims, r, 1.0,
                   plan=xt.make_plan(XB.METHOD_TTGT))
        got = _run(xt, dev, xt.tensor_contract_noalloc, pattern, dtk, ddims, d, ldims, l, rdims, r, 1.0)
        assert np.array_equal(got.view(np.uint8), ref.view(np.uint8)), pattern


def test_noalloc_allocates_nothing(xt, dev):
    """After a first call (which may load GPU code), two more calls leave the
    device's free memory and its stream-ordered pool's high-water mark as they were."""
    import torch
    from cuda.bindings import driver as cu
    ok = cu.CUresult.CUDA_SUCCESS
    assert cu.cuInit(0)[0] == ok
    pattern, ext, dtk = CASES[0]
    ddims, ldims, rdims, d, l, r = _inputs(pattern, ext, dtk, 3)
    dd, ld, rd = dev.put(d), dev.put(l), dev.put(r)
    args = (pattern, dtk, ddims, dd.data_ptr(), ldims, ld.data_ptr(), rdims, rd.data_ptr(), 1.0)
    xt.tensor_contract_noalloc(*args, stream=dev.stream())
    torch.cuda.synchronize()
    err, pool = cu.cuDeviceGetDefaultMemPool(torch.cuda.current_device())
    assert err == ok
    high = cu.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH
    assert cu.cuMemPoolSetAttribute(pool, high, cu.cuuint64_t(0))[0] == ok
    err, high0 = cu.cuMemPoolGetAttribute(pool, high)
    err, free0, _ = cu.cuMemGetInfo()
    for _ in range(2):
        xt.tensor_contract_noalloc(*args, stream=dev.stream())
    torch.cuda.synchronize()
    err, high1 = cu.cuMemPoolGetAttribute(pool, high)
    err, free1, _ = cu.cuMemGetInfo()
    assert int(high1) == int(high0)
    assert free1 == free0
    xt.device_check(dev.stream())


def test_noalloc_rejects_requests_over_the_limit(xt, dev):
    """8 * (M*K + N*K + M*N) bytes over 64 MiB: TB_ERR_LIMIT, nothing launched, D untouched."""
    pattern = "D(i,j)+=L(k,i)*R(k,j)"
    # M = N = 2048, K = 1024 needs exactly 64 MiB; one more column of R does not fit.
    ddims, ldims, rdims = [2048, 2049], [1024, 2048], [1024, 2049]
    d = np.full(2048 * 2049, 3.0)
    dd = dev.put(d)
    ld = dev.empty(1024 * 2048 * 8, fill=0)
    rd = dev.empty(1024 * 2049 * 8, fill=0)
    before = xt.launch_count()
    with pytest.raises(XB.TBError) as ei:
        xt.tensor_contract_noalloc(pattern, O.R8, ddims, dd.data_ptr(), ldims, ld.data_ptr(), rdims,
                                   rd.data_ptr(), 1.0, stream=dev.stream())
    assert ei.value.code == 7 and "static scratch array" in str(ei.value)
    assert xt.launch_count() == before
    assert np.array_equal(dev.get(dd, np.float64, d.size), d)
    # the exact fit is accepted
    ddims, rdims = [2048, 2048], [1024, 2048]
    got = _run(xt, dev, xt.tensor_contract_noalloc, pattern, O.R8, ddims, np.zeros(2048 * 2048), ldims,
               np.full(1024 * 2048, 0.5), rdims, np.full(1024 * 2048, 0.25), 1.0)
    assert np.all(got == 1024 * 0.125)
