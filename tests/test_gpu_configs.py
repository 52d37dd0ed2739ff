"""GPU parity on the configured workloads, against the oracle:

  C1  the single-block 40^4 R8 contraction D(a,b,c,d) += 0.5 * L(c,k,a,l) *
      R(l,d,k,b) with L and R from one seeded stream (seed 0, L first), D = 0,
      by every method, against the double-double oracle over the whole tensor
      (TALSH/test.cpp:1016-1110 runs the same contraction through
      gpu_tensor_block_contract_dlf);
  C2  one 256 MiB case of every class of the permutation sweep (R8/R4, ranks
      2-6, uniform and skewed extents) bit for bit against oracle.permute on
      the host, and the add sweep's classes against oracle.tensor_add
      (TALSH/tensor_algebra_cpu.F90:3151, :3312);
  C3  the six CCSD-like configurations at reduced extents (v = 48, o = 12, same
      patterns and data kinds), METHOD_AUTO against the double-double oracle
      over the whole output tensor.

Tolerances (relative Frobenius vs double-double): 1e-12 for R8/C8 on the
tensor cores, 1e-13 for plain FP64 TTGT, 1e-4 for R4/C4 (split-BF16), 2e-5
for plain FP32.  Permutations and adds: bit-exact."""
import numpy as np
import pytest

import bench
import exatensor_b200 as XB
import oracle as O
from tests.test_gpu_contract import oracle_dd

pytestmark = pytest.mark.gpu
TOL = {(XB.METHOD_FUSED, O.R8): 1e-12, (XB.METHOD_FUSED, O.C8): 1e-12, (XB.METHOD_FUSED, O.R4): 1e-4,
       (XB.METHOD_FUSED, O.C4): 1e-4, (XB.METHOD_TTGT, O.R8): 1e-13, (XB.METHOD_TTGT, O.C8): 1e-13,
       (XB.METHOD_TTGT, O.R4): 2e-5, (XB.METHOD_TTGT, O.C4): 2e-5}


@pytest.mark.parametrize("method", [XB.METHOD_AUTO, XB.METHOD_TTGT, XB.METHOD_FUSED])
def test_c1_seeded_single_block_contraction(xt, dev, method):
    pat = "D(a,b,c,d)+=L(c,k,a,l)*R(l,d,k,b)"
    dims, vol = [40] * 4, 40 ** 4
    u = O.splitmix64_uniform(2 * vol, 0)
    L, R, D = u[:vol].copy(), u[vol:].copy(), np.zeros(vol)
    ref = oracle_dd(pat, D, dims, L, dims, R, dims, 0.5, True)
    dd, ld, rd = dev.put(D), dev.put(L), dev.put(R)
    xt.tensor_contract(pat, O.R8, dims, dd.data_ptr(), dims, ld.data_ptr(), dims, rd.data_ptr(), 0.5,
                       plan=xt.make_plan(method), stream=dev.stream())
    got = dev.get(dd, np.float64, vol)
    st = xt.last_contract_stats()
    assert st.m == 1600 and st.k == 1600
    err = O.rel_frobenius(got, ref)
    assert err <= TOL[(st.method, O.R8)], (st.method, err)


def first_of_each_class(cases):
    seen, out = set(), []
    for c in cases:
        if c["cls"] not in seen:
            seen.add(c["cls"])
            out.append(c)
    return out


@pytest.mark.parametrize("case", first_of_each_class(bench.sweep_cases()), ids=lambda c: c["cls"])
def test_c2_sweep_class_bit_exact_at_full_size(xt, dev, case):
    import torch
    dtk, dims, perm = case["dtk"], case["dims"], case["perm"]
    n = bench.vol(dims)
    es = 8 if dtk == O.R8 else 4
    a = torch.empty(n * es, dtype=torch.uint8, device="cuda")
    b = torch.empty_like(a)
    xt.fill_uniform(dtk, n, a.data_ptr(), 3, stream=dev.stream())
    xt.tensor_copy(dtk, dims, perm, a.data_ptr(), b.data_ptr(), 0, dev.stream())
    x = dev.get(a, O.NP_DTYPE[dtk], n)
    got = dev.get(b, O.NP_DTYPE[dtk], n)
    assert np.array_equal(got.view(np.uint8), O.permute(x, dims, list(perm)).view(np.uint8)), (dims, perm)


@pytest.mark.parametrize("cls", ["r8_4", "r4_4", "r8_6", "r4_6"])
def test_c2_add_class_bit_exact_at_full_size(xt, dev, cls):
    import torch
    case = [c for c in bench.add_cases() if c["cls"] == cls][5]
    dtk, dims, perm = case["dtk"], case["dims"], case["perm"]
    n = bench.vol(dims)
    es = 8 if dtk == O.R8 else 4
    l = torch.empty(n * es, dtype=torch.uint8, device="cuda")
    d = torch.empty_like(l)
    xt.fill_uniform(dtk, n, l.data_ptr(), 4, stream=dev.stream())
    xt.fill_uniform(dtk, n, d.data_ptr(), 5, stream=dev.stream())
    lh = dev.get(l, O.NP_DTYPE[dtk], n).copy()
    d0 = dev.get(d, O.NP_DTYPE[dtk], n).copy()
    xt.tensor_add(dtk, dims, perm, d.data_ptr(), l.data_ptr(), 0.37, 0, dev.stream())
    got = dev.get(d, O.NP_DTYPE[dtk], n)
    ref = O.tensor_add(list(perm), d0, lh, dims, 0.37)
    assert np.array_equal(got.view(np.uint8), ref.view(np.uint8)), (dims, perm)


@pytest.mark.parametrize("name", list(bench.WORKLOADS))
def test_c3_ccsd_configs_reduced_whole_tensor(xt, dev, name):
    import torch
    wl = dict(bench.WORKLOADS[name])
    wl["v"], wl["o"] = 48, 12
    dtk = wl["dtk"]
    ddims, ldims, rdims = bench.shapes(wl["pattern"], wl["v"], wl["o"])
    dt = O.NP_DTYPE[dtk]
    cplx = dtk in (O.C4, O.C8)

    def data(n, seed):
        x = O.splitmix64_uniform(n * (2 if cplx else 1), seed)
        return (x[0::2] + 1j * x[1::2] if cplx else x).astype(dt)
    L = (data(bench.vol(ldims), 1) / wl["v"]).astype(dt)
    R = data(bench.vol(rdims), 2)
    D = np.zeros(bench.vol(ddims), dtype=dt)
    ref = oracle_dd(wl["pattern"], D, ddims, L, ldims, R, rdims, 1.0, True)
    for method in (XB.METHOD_AUTO, XB.METHOD_TTGT):
        dd, ld, rd = dev.put(D), dev.put(L), dev.put(R)
        xt.tensor_contract(wl["pattern"], dtk, ddims, dd.data_ptr(), ldims, ld.data_ptr(), rdims, rd.data_ptr(),
                           1.0, plan=xt.make_plan(method), stream=dev.stream())
        got = dev.get(dd, dt, D.size)
        st = xt.last_contract_stats()
        err = O.rel_frobenius(got, ref)
        assert err <= TOL[(st.method, dtk)], (name, st.method, err)
    torch.cuda.synchronize()
