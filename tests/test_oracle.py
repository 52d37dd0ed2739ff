"""The CPU oracle pinned against the reference's own known answers.

Every expectation here comes from the reference: the closed-form values its
test drivers print (TALSH/test.cpp, TALSH/main.F90), digital patterns and
TTGT permutations derived by hand from TALSH/tensor_algebra_cpu.F90, and the
48-pattern corpus TALSH/tensor_contractions.txt (tests/golden/).
"""
import json
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
KATS = json.load(open(os.path.join(GOLD, "kats.json")))
CTM = json.load(open(os.path.join(GOLD, "ctm_patterns.json")))["entries"]
DTK = {"R4": O.R4, "R8": O.R8, "C4": O.C4, "C8": O.C8}


@pytest.mark.parametrize("case", KATS["patterns"], ids=lambda c: c["pattern"])
def test_parse_pattern_kat(case):
    cptrn, d, l, r, cj = O.parse_pattern(case["pattern"])
    assert cptrn == case["cptrn"]
    assert [d, l, r] == case["ranks"]
    assert cj == case["conj"]


@pytest.mark.parametrize("case", KATS["pattern_errors"], ids=lambda c: c["pattern"] or "empty")
def test_parse_pattern_errors(case):
    with pytest.raises(O.PatternError) as ei:
        O.parse_pattern(case["pattern"])
    assert ei.value.code == case["code"]


@pytest.mark.parametrize("case", KATS["permutations"], ids=lambda c: str(c["cptrn"]))
def test_contr_permutations_kat(case):
    dprm, lprm, rprm, ncd, nlu, nru = O.contr_permutations(case["cptrn"], case["lrank"], case["rrank"],
                                                           case["conj"])
    assert (dprm, lprm, rprm) == (case["dprm"], case["lprm"], case["rprm"])
    assert (ncd, nlu, nru) == (case["ncd"], case["nlu"], case["nru"])


@pytest.mark.parametrize("entry", CTM, ids=lambda e: e["pattern"])
def test_ctm_corpus_parses_consistently(entry):
    """Every corpus pattern parses, its shapes agree with the digital pattern,
    and the TTGT permutations are valid permutations."""
    cptrn, d, l, r, cj = O.parse_pattern(entry["pattern"])
    assert (d, l, r) == (len(entry["ddims"]), len(entry["ldims"]), len(entry["rdims"]))
    for i, c in enumerate(cptrn):
        ext = entry["ldims"][i] if i < l else entry["rdims"][i - l]
        if c > 0:
            assert entry["ddims"][c - 1] == ext
        else:
            other = entry["rdims"] if i < l else entry["ldims"]
            assert other[-c - 1] == ext
    dprm, lprm, rprm, ncd, nlu, nru = O.contr_permutations(cptrn, l, r)
    assert sorted(dprm) == list(range(1, d + 1))
    assert sorted(lprm) == list(range(1, l + 1))
    assert sorted(rprm) == list(range(1, r + 1))
    assert nlu + nru == d


def _np_permute(flat, dims, o2n):
    """numpy restatement of an O2N permutation in dlf layout."""
    a = flat.reshape(dims, order="F")
    n2o = [0] * len(dims)
    for i, p in enumerate(o2n):
        n2o[p - 1] = i
    return np.ascontiguousarray(a.transpose(n2o)).ravel(order="F") if len(dims) else flat.copy()


@pytest.mark.parametrize("dtk", [O.R4, O.R8, O.C4, O.C8])
def test_permute_all_rank4(dtk):
    import itertools
    dims = [3, 4, 5, 2]
    rng = np.random.default_rng(1)
    vol = int(np.prod(dims))
    x = rng.uniform(-1, 1, vol)
    if dtk in (O.C4, O.C8):
        x = x + 1j * rng.uniform(-1, 1, vol)
    x = x.astype(O.NP_DTYPE[dtk])
    for perm in itertools.permutations([1, 2, 3, 4]):
        out = O.permute(x, dims, perm)
        assert np.array_equal(out.view(np.uint8), _np_permute(x, dims, perm).view(np.uint8))
        outb = O.permute_blocked(x, dims, perm)
        assert np.array_equal(outb.view(np.uint8), out.view(np.uint8))


def test_permute_conj_and_roundtrip():
    dims = [7, 1, 6, 5, 3]
    rng = np.random.default_rng(2)
    vol = int(np.prod(dims))
    x = (rng.uniform(-1, 1, vol) + 1j * rng.uniform(-1, 1, vol)).astype(np.complex128)
    o2n = [3, 5, 1, 2, 4]
    y = O.permute(x, dims, o2n, conj=True)
    assert np.array_equal(y, np.conj(_np_permute(x, dims, o2n)))
    inv = [0] * 5
    for i, p in enumerate(o2n):
        inv[p - 1] = i + 1
    z = O.permute(y, O.permuted_dims(dims, o2n), inv, conj=True)
    assert np.array_equal(z, x)


def test_add_semantics_two_roundings():
    """d = d + l*a with two roundings (no FMA), R4 scale rounded to float first."""
    rng = np.random.default_rng(3)
    d = rng.uniform(-1, 1, 1000).astype(np.float32)
    l = rng.uniform(-1, 1, 1000).astype(np.float32)
    a = 0.3
    ref = d + (l * np.float32(a))
    O.add(d, l, a)
    assert np.array_equal(d, ref)
    d8 = rng.uniform(-1, 1, 1000)
    l8 = rng.uniform(-1, 1, 1000)
    ref8 = d8 + l8 * 0.7
    O.add(d8, l8, 0.7)
    assert np.array_equal(d8, ref8)
    # complex: textbook product, conjugated left operand via conj bit 1
    dc = (rng.uniform(-1, 1, 100) + 1j * rng.uniform(-1, 1, 100))
    lc = (rng.uniform(-1, 1, 100) + 1j * rng.uniform(-1, 1, 100))
    s = 0.25 - 0.5j
    lcc = np.conj(lc)
    re = lcc.real * s.real - lcc.imag * s.imag
    im = lcc.real * s.imag + lcc.imag * s.real
    ref_c = dc + (re + 1j * im)
    O.add(dc, lc, s, conj_bits=2)
    assert np.array_equal(dc, ref_c)


def test_scale_real_of_complex_factor():
    """Real data takes cmplx8_to_real8 of the factor (tensor_algebra_cpu.F90:430)."""
    d = np.ones(4)
    O.scale(d, -3.0 + 4.0j)
    assert np.allclose(d, -5.0)
    d = np.ones(4)
    O.scale(d, 0.0 + 2.0j)
    assert np.allclose(d, 2.0)


def _kat_tensors(case):
    dt = O.NP_DTYPE[DTK[case["dtype"]]]
    mk = lambda dims, v: np.full(int(np.prod(dims)) if dims else 1, v, dtype=dt)
    return mk(case["ddims"], case["dinit"]), mk(case["ldims"], case["linit"]), mk(case["rdims"], case["rinit"])


@pytest.mark.parametrize("case", KATS["contractions"], ids=lambda c: c["name"])
@pytest.mark.parametrize("mode", [0, 1])
def test_contraction_kats(case, mode):
    cptrn, _, _, _, cj = O.parse_pattern(case["pattern"])
    d, l, r = _kat_tensors(case)
    O.contract(cptrn, d, case["ddims"], l, case["ldims"], r, case["rdims"], alpha=case["alpha"],
               conj_bits=cj, accumulative=case["accumulative"], mode=mode)
    if d.dtype in (np.float32, np.complex64):
        # sequential FP32 sums (mode 0) drift ~K*eps; double-double (mode 1) only
        # carries the float rounding of the input constants
        tol = 1e-3 if mode == 0 else 1e-6
    else:
        tol = 1e-12
    assert np.allclose(d, case["element"], rtol=tol, atol=0)
    ntol = max(tol, 1e-9)  # the norm is a long sequential sum of equal terms
    if "norm1" in case:
        assert abs(O.norm1(d) - case["norm1"]) <= ntol * case["norm1"]
    if "norm2sq" in case:
        assert abs(O.norm2sq(d) - case["norm2sq"]) <= ntol * case["norm2sq"]


def test_explicit_loop_check():
    """TALSH/test.cpp:895-1000: contract with alpha=-2 then alpha=+1, add L*R by
    explicit loops; the destination returns to ~0."""
    e = KATS["explicit_loop"]
    cptrn, *_ = O.parse_pattern(e["pattern"])
    d0, d1 = e["ddims"]; l0, l1 = e["ldims"]; r0, r1, r2, r3 = e["rdims"]
    rng = np.random.default_rng(7)
    L = 1e6 / (rng.integers(0, 2**31 - 1, l0 * l1) + 1.0)
    R = 1e5 / (rng.integers(0, 2**31 - 1, r0 * r1 * r2 * r3) + 1.0)
    D = np.zeros(d0 * d1)
    for a in e["alphas"]:
        O.contract(cptrn, D, e["ddims"], L, e["ldims"], R, e["rdims"], alpha=a)
    scale = np.abs(D).sum()
    for ib in range(d1):
        for ia in range(d0):
            for idd in range(l1):
                for ic in range(l0):
                    D[ia + ib * d0] += L[ic + idd * l0] * R[idd + ia * r0 + ib * r1 * r0 + ic * r2 * r1 * r0]
    assert np.abs(D).sum() <= 1e-13 * scale


def test_dd_oracle_matches_numpy_einsum():
    rng = np.random.default_rng(11)
    pat = "D(a,b,c,d)+=L(c,k,a,l)*R(l,d,k,b)"
    cptrn, *_ = O.parse_pattern(pat)
    n = 6
    L = rng.uniform(-1, 1, n ** 4)
    R = rng.uniform(-1, 1, n ** 4)
    D = rng.uniform(-1, 1, n ** 4)
    ref = D.reshape([n] * 4, order="F") + 0.5 * np.einsum(
        "ckal,ldkb->abcd", L.reshape([n] * 4, order="F"), R.reshape([n] * 4, order="F"))
    for mode in (0, 1):
        out = D.copy()
        O.contract(cptrn, out, [n] * 4, L, [n] * 4, R, [n] * 4, alpha=0.5, mode=mode)
        assert np.allclose(out, ref.ravel(order="F"), rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("dtk", [O.C4, O.C8])
def test_complex_contraction_conj(dtk):
    rng = np.random.default_rng(12)
    pat = "D+(a,b)+=L(c,a)*R+(c,b)"   # conj(D) += L * conj(R)  ->  D += conj(L) * R
    cptrn, _, _, _, cj = O.parse_pattern(pat)
    m, k, n = 5, 7, 3
    L = (rng.uniform(-1, 1, k * m) + 1j * rng.uniform(-1, 1, k * m)).astype(O.NP_DTYPE[dtk])
    R = (rng.uniform(-1, 1, k * n) + 1j * rng.uniform(-1, 1, k * n)).astype(O.NP_DTYPE[dtk])
    D = np.zeros(m * n, dtype=O.NP_DTYPE[dtk])
    O.contract(cptrn, D, [m, n], L, [k, m], R, [k, n], alpha=1.0, conj_bits=cj, mode=1)
    ref = np.conj(L.reshape(k, m, order="F")).T @ R.reshape(k, n, order="F")
    tol = 1e-5 if dtk == O.C4 else 1e-13
    assert np.allclose(D.reshape(m, n, order="F"), ref, rtol=tol, atol=tol)


def test_splitmix_uniform_range_and_determinism():
    x = O.splitmix64_uniform(100000, 0)
    assert x.min() >= -1.0 and x.max() < 1.0
    assert np.array_equal(x, O.splitmix64_uniform(100000, 0))
    assert abs(x.mean()) < 0.01


def test_blas_baseline_matches_oracle():
    if not O.blas_available():
        pytest.skip("bundled OpenBLAS not found")
    rng = np.random.default_rng(5)
    pat = "D(a,b,c,d)+=L(c,k,a,l)*R(l,d,k,b)"
    cptrn, *_ = O.parse_pattern(pat)
    n = 9
    L = rng.uniform(-1, 1, n ** 4); R = rng.uniform(-1, 1, n ** 4); D = rng.uniform(-1, 1, n ** 4)
    a = D.copy(); b = D.copy()
    O.contract(cptrn, a, [n] * 4, L, [n] * 4, R, [n] * 4, alpha=0.5, mode=1)
    O.contract_blas(cptrn, b, [n] * 4, L, [n] * 4, R, [n] * 4, alpha=0.5)
    assert O.rel_frobenius(b, a) < 1e-14


def test_reference_nvtal_library_loads():
    """The reference's own NV-TAL kernels (oracle/_ref, built from the
    reference's sources by `make -C oracle ref`) load on the CPU and export the
    harness's entry points; the GPU parity test calls them."""
    import ctypes
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                        "libnvtal_ref.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref/libnvtal_ref.so not built (needs the reference sources)")
    lib = ctypes.CDLL(path)
    for name in ("ref_init", "ref_copy", "ref_add", "ref_contract", "gpu_tensor_block_copy",
                 "gpu_tensor_block_add", "gpu_tensor_block_contract_dlf", "get_contr_permutations"):
        assert hasattr(lib, name), name
