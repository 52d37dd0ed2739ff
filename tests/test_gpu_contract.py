"""GPU parity: tensor contractions (tb_tensor_contract) against the oracle's
restatement of tensor_block_contract (TALSH/tensor_algebra_cpu.F90:3675) with
double-double accumulation (the FP64 error oracle).

Tolerances (relative Frobenius error vs the double-double oracle):
  plain TTGT:  R8/C8 1e-13, R4/C4 2e-5 (FP32 accumulation over K <= 4096)
  fused:       R8/C8 1e-12 (INT8 slices), R4/C4 1e-4 (3-term split-BF16)
The closed-form known answers of the reference's tests must hold to the same
bounds."""
import json
import os
import random

import numpy as np
import pytest

import exatensor_b200 as XB
import oracle as O
from tests.test_gpu_permute import rand_host

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
KATS = json.load(open(os.path.join(GOLD, "kats.json")))
CTM = json.load(open(os.path.join(GOLD, "ctm_patterns.json")))["entries"]
DTK = {"R4": O.R4, "R8": O.R8, "C4": O.C4, "C8": O.C8}
TOL = {(XB.METHOD_TTGT, O.R8): 1e-13, (XB.METHOD_TTGT, O.C8): 1e-13, (XB.METHOD_TTGT, O.R4): 2e-5,
       (XB.METHOD_TTGT, O.C4): 2e-5, (XB.METHOD_FUSED, O.R8): 1e-12, (XB.METHOD_FUSED, O.C8): 1e-12,
       (XB.METHOD_FUSED, O.R4): 1e-4, (XB.METHOD_FUSED, O.C4): 1e-4,
       (XB.METHOD_AUTO, O.R8): 1e-12, (XB.METHOD_AUTO, O.C8): 1e-12, (XB.METHOD_AUTO, O.R4): 1e-4,
       (XB.METHOD_AUTO, O.C4): 1e-4}
METHODS = [XB.METHOD_TTGT, XB.METHOD_AUTO]


def run_gpu(xt, dev, pattern, d, ddims, l, ldims, r, rdims, alpha, accumulative, method):
    dd, ld, rd = dev.put(d), dev.put(l), dev.put(r)
    dtk = O.DTK_OF[d.dtype]
    xt.tensor_contract(pattern, dtk, ddims, dd.data_ptr(), ldims, ld.data_ptr(), rdims, rd.data_ptr(), alpha,
                       accumulative=accumulative, plan=xt.make_plan(method), stream=dev.stream())
    return dev.get(dd, d.dtype, d.size)


def oracle_dd(pattern, d, ddims, l, ldims, r, rdims, alpha, accumulative):
    cptrn, _, _, _, cj = O.parse_pattern(pattern)
    out = d.copy()
    O.contract(cptrn, out, ddims, l, ldims, r, rdims, alpha, cj, accumulative, mode=1)
    return out


@pytest.mark.parametrize("case", KATS["contractions"], ids=lambda c: c["name"])
@pytest.mark.parametrize("method", METHODS)
def test_reference_known_answers(xt, dev, case, method):
    dtk = DTK[case["dtype"]]
    dt = O.NP_DTYPE[dtk]
    mk = lambda dims, v: np.full(int(np.prod(dims)) if dims else 1, v, dtype=dt)
    d = mk(case["ddims"], case["dinit"])
    got = run_gpu(xt, dev, case["pattern"], d, case["ddims"], mk(case["ldims"], case["linit"]), case["ldims"],
                  mk(case["rdims"], case["rinit"]), case["rdims"], case["alpha"], case["accumulative"], method)
    tol = 1e-4 if dtk in (O.R4, O.C4) else 1e-12
    assert np.allclose(got, case["element"], rtol=tol, atol=0)
    if "norm1" in case:
        assert abs(O.norm1(got) - case["norm1"]) <= max(tol, 1e-9) * case["norm1"]


RANDOM_PATTERNS = [
    ("D(a,b,c,d)+=L(c,k,a,l)*R(l,d,k,b)", {"a": 9, "b": 7, "c": 8, "d": 6, "k": 10, "l": 5}),
    ("D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)", {"a": 12, "b": 12, "c": 12, "d": 12, "i": 5, "j": 5}),
    ("D(a,i,b,j)+=L(a,k,c,i)*R(c,b,k,j)", {"a": 10, "b": 10, "c": 10, "i": 6, "j": 6, "k": 6}),
    ("D(i,j)+=L(k,i)*R(k,j)", {"i": 131, "j": 77, "k": 300}),
    ("D(i,j)+=L(i,k)*R(j,k)", {"i": 64, "j": 96, "k": 128}),
    ("D(a,b,c)+=L(b,d,a)*R(d,c)", {"a": 20, "b": 17, "c": 9, "d": 33}),
    ("D(a,b)+=L(a)*R(b)", {"a": 300, "b": 257}),
    ("D(a,b,c)+=L(c,a,b)*R()", {"a": 7, "b": 8, "c": 9}),
    ("D(b)+=L(k,l)*R(l,b,k)", {"b": 37, "k": 19, "l": 23}),
]


def shapes(pattern, ext):
    import re
    groups = re.findall(r"\(([^)]*)\)", pattern)
    return [[ext[x] for x in g.split(",") if x] for g in groups]


@pytest.mark.parametrize("dtk", [O.R8, O.C8, O.R4, O.C4])
@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("pi", range(len(RANDOM_PATTERNS)))
def test_random_contractions_vs_fp64_oracle(xt, dev, dtk, method, pi):
    pattern, ext = RANDOM_PATTERNS[pi]
    ddims, ldims, rdims = shapes(pattern, ext)
    vol = lambda s: int(np.prod(s)) if s else 1
    d = rand_host(dtk, vol(ddims), 1 + pi)
    l = rand_host(dtk, vol(ldims), 2 + pi)
    r = rand_host(dtk, vol(rdims), 3 + pi)
    for accumulative, alpha in ((True, 0.5), (False, -1.25 + (0.5j if dtk in (O.C4, O.C8) else 0))):
        ref = oracle_dd(pattern, d, ddims, l, ldims, r, rdims, alpha, accumulative)
        got = run_gpu(xt, dev, pattern, d, ddims, l, ldims, r, rdims, alpha, accumulative, method)
        err = O.rel_frobenius(got, ref)
        assert err <= TOL[(method, dtk)], (pattern, accumulative, err)


@pytest.mark.parametrize("dtk", [O.C4, O.C8])
@pytest.mark.parametrize("pattern", ["D(a,b)+=L+(k,a)*R(k,b)", "D(a,b)+=L(k,a)*R+(k,b)", "D+(a,b)+=L(k,a)*R(k,b)",
                                     "D()+=L+(a,k)*R(k,a)"])
@pytest.mark.parametrize("method", METHODS)
def test_complex_conjugation(xt, dev, dtk, pattern, method):
    ext = {"a": 33, "b": 21, "k": 40}
    ddims, ldims, rdims = shapes(pattern, ext)
    vol = lambda s: int(np.prod(s)) if s else 1
    d, l, r = rand_host(dtk, vol(ddims), 1), rand_host(dtk, vol(ldims), 2), rand_host(dtk, vol(rdims), 3)
    ref = oracle_dd(pattern, d, ddims, l, ldims, r, rdims, 0.7 - 0.2j, True)
    got = run_gpu(xt, dev, pattern, d, ddims, l, ldims, r, rdims, 0.7 - 0.2j, True, method)
    assert O.rel_frobenius(got, ref) <= TOL[(method, dtk)]


def test_ctm_corpus_reduced_extents(xt, dev):
    """All 48 patterns of TALSH/tensor_contractions.txt with extents scaled down
    so the double-double oracle finishes quickly (R8, both methods)."""
    for e in CTM:
        pattern = e["pattern"]
        labels = {}
        import re
        groups = re.findall(r"\(([^)]*)\)", pattern)
        for g, dims in zip(groups, (e["ddims"], e["ldims"], e["rdims"])):
            for x, n in zip(g.split(","), dims):
                labels[x] = max(2, min(n, 11) if n > 11 else n) if n < 30 else 9
        ddims, ldims, rdims = shapes(pattern, labels)
        vol = lambda s: int(np.prod(s)) if s else 1
        d, l, r = rand_host(O.R8, vol(ddims), 1), rand_host(O.R8, vol(ldims), 2), rand_host(O.R8, vol(rdims), 3)
        ref = oracle_dd(pattern, d, ddims, l, ldims, r, rdims, 1.0, True)
        for method in METHODS:
            got = run_gpu(xt, dev, pattern, d, ddims, l, ldims, r, rdims, 1.0, True, method)
            assert O.rel_frobenius(got, ref) <= TOL[(method, O.R8)], (pattern, method)


def test_explicit_loop_check(xt, dev):
    """TALSH/test.cpp:895-1000 on the GPU: alpha=-2 then +1, then explicit loops."""
    e = KATS["explicit_loop"]
    d0, d1 = e["ddims"]; l0, l1 = e["ldims"]; r0, r1, r2, r3 = e["rdims"]
    rng = np.random.default_rng(7)
    L = 1e6 / (rng.integers(0, 2**31 - 1, l0 * l1) + 1.0)
    R = 1e5 / (rng.integers(0, 2**31 - 1, r0 * r1 * r2 * r3) + 1.0)
    D = np.zeros(d0 * d1)
    for a in e["alphas"]:
        D = run_gpu(xt, dev, e["pattern"], D, e["ddims"], L, e["ldims"], R, e["rdims"], a, True, XB.METHOD_TTGT)
    scale = np.abs(D).sum()
    for ib in range(d1):
        for ia in range(d0):
            for idd in range(l1):
                for ic in range(l0):
                    D[ia + ib * d0] += L[ic + idd * l0] * R[idd + ia * r0 + ib * r1 * r0 + ic * r2 * r1 * r0]
    assert np.abs(D).sum() <= 1e-13 * scale


def test_errors_are_reported(xt, dev):
    d = dev.empty(64); l = dev.empty(64); r = dev.empty(64)
    with pytest.raises(XB.TBError):   # shapes do not match the pattern
        xt.tensor_contract("D(a,b)+=L(k,a)*R(k,b)", O.R8, [2, 2], d.data_ptr(), [3, 2], l.data_ptr(), [2, 2],
                           r.data_ptr(), stream=dev.stream())
    with pytest.raises(XB.TBError):   # hyper-index
        xt.tensor_contract("D(a,b)+=L(a,k,b)*R(k,b)", O.R8, [2, 2], d.data_ptr(), [2, 2, 2], l.data_ptr(), [2, 2],
                           r.data_ptr(), stream=dev.stream())
    with pytest.raises(XB.TBError):   # bad data kind
        xt.tensor_contract("D(a,b)+=L(k,a)*R(k,b)", 5, [2, 2], d.data_ptr(), [2, 2], l.data_ptr(), [2, 2],
                           r.data_ptr(), stream=dev.stream())
