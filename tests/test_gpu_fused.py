"""GPU parity of the tensor-core contraction (TB_METHOD_FUSED): FP64 (R8/C8)
by modular residues or INT8 slices and FP32 (R4/C4) by split BF16 through
tcgen05, against the double-double FP64 oracle.

Tolerances (relative Frobenius error vs the oracle), stated per data kind:
  R8/C8: 1e-12 with the default residues or 6 slices (the FP64 accuracy target)
  R4/C4: 1e-4  (3-term split-BF16; its products keep about 16 mantissa bits)
"""
import numpy as np
import pytest

import exatensor_b200 as XB
import oracle as O
from tests.test_gpu_contract import oracle_dd, run_gpu, shapes
from tests.test_gpu_permute import rand_host

pytestmark = pytest.mark.gpu
TOL = {O.R8: 1e-12, O.C8: 1e-12, O.R4: 1e-4, O.C4: 1e-4}


def fused(xt, dev, pattern, ext, dtk, alpha=1.0, accumulative=True, plan=None, seed=1):
    ddims, ldims, rdims = shapes(pattern, ext)
    vol = lambda s: int(np.prod(s)) if s else 1
    d, l, r = rand_host(dtk, vol(ddims), seed), rand_host(dtk, vol(ldims), seed + 1), rand_host(dtk, vol(rdims), seed + 2)
    ref = oracle_dd(pattern, d, ddims, l, ldims, r, rdims, alpha, accumulative)
    dd, ld, rd = dev.put(d), dev.put(l), dev.put(r)
    xt.tensor_contract(pattern, dtk, ddims, dd.data_ptr(), ldims, ld.data_ptr(), rdims, rd.data_ptr(), alpha,
                       accumulative=accumulative, plan=plan or xt.make_plan(XB.METHOD_FUSED), stream=dev.stream())
    got = dev.get(dd, d.dtype, d.size)
    xt.device_check(dev.stream())
    st = xt.last_contract_stats()
    assert st.method == XB.METHOD_FUSED
    return O.rel_frobenius(got, ref), st


def test_fused_r8_square(xt, dev):
    # the default for R8 on the tensor cores: modular residues (Ozaki scheme II)
    err, st = fused(xt, dev, "D(i,j)+=L(k,i)*R(k,j)", {"i": 256, "j": 256, "k": 256}, O.R8)
    assert err <= TOL[O.R8], err
    assert st.moduli >= 8 and st.residue_bits >= 46 and st.products == st.moduli and st.passes == st.moduli
    # INT8 slices (Ozaki scheme I) on request
    err, st = fused(xt, dev, "D(i,j)+=L(k,i)*R(k,j)", {"i": 256, "j": 256, "k": 256}, O.R8,
                    plan=xt.make_plan(XB.METHOD_FUSED, moduli=-1))
    assert err <= TOL[O.R8], err
    assert st.moduli == 0 and st.slices == 6 and st.passes >= 6 and st.products == 21


@pytest.mark.parametrize("dtk,bits,K", [(O.R8, 20, 4096), (O.C8, 19, 4096), (O.R8, 16, 200000)])
def test_residue_path_is_exact_on_integer_data(xt, dev, dtk, bits, K):
    """Integer operands of up to `bits` bits: every step of the residue path is
    exact (the row scaling keeps the integers, the residues are the integers'
    residues, the INT8 products are exact, the CRT recovers the exact sum), so
    D must equal the integer product bit for bit.  K = 200000 is longer than
    one exact INT32 pass: its residues come from two K chunks added mod m."""
    rng = np.random.default_rng(4)
    M, N = (512, 384) if K <= 4096 else (128, 96)
    ints = lambda n: rng.integers(-(2 ** bits), 2 ** bits + 1, size=n)
    if dtk == O.R8:
        l, r = ints(K * M).astype(np.float64), ints(K * N).astype(np.float64)
        ref = l.astype(np.int64).reshape(M, K) @ r.astype(np.int64).reshape(N, K).T
        want = ref.astype(np.float64).T.ravel()  # D(i,j), i fastest
    else:
        l = ints(K * M) + 1j * ints(K * M)
        r = ints(K * N) + 1j * ints(K * N)
        lr, li = l.real.astype(np.int64).reshape(M, K), l.imag.astype(np.int64).reshape(M, K)
        rr, ri = r.real.astype(np.int64).reshape(N, K), r.imag.astype(np.int64).reshape(N, K)
        re, im = lr @ rr.T - li @ ri.T, lr @ ri.T + li @ rr.T
        want = (re.astype(np.float64) + 1j * im.astype(np.float64)).T.ravel()
    # L(k,i) with k fastest: row i of the matrix above is contiguous along k
    d = np.zeros(M * N, dtype=want.dtype)
    dd, ld, rd = dev.put(d), dev.put(l), dev.put(r)
    xt.tensor_contract("D(i,j)+=L(k,i)*R(k,j)", dtk, [M, N], dd.data_ptr(), [K, M], ld.data_ptr(), [K, N],
                       rd.data_ptr(), 1.0, accumulative=False, plan=xt.make_plan(XB.METHOD_FUSED), stream=dev.stream())
    got = dev.get(dd, d.dtype, d.size)
    xt.device_check(dev.stream())
    st = xt.last_contract_stats()
    assert st.method == XB.METHOD_FUSED and st.moduli >= 8
    assert st.passes == st.moduli * (1 if K <= 4096 else 2)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("dtk", [O.R8, O.C8])
@pytest.mark.parametrize("moduli", [10, 12, 14, 15])
def test_residue_moduli_counts(xt, dev, dtk, moduli):
    """More moduli keep more bits per operand (p, with prod m_i > 2 K 2^(2p));
    the error falls with p: it stays within 2^(5-p) relative Frobenius
    (uniform data, K = 512) for every count."""
    ext = {"i": 192, "j": 160, "k": 512}
    err, st = fused(xt, dev, "D(i,j)+=L(k,i)*R(k,j)", ext, dtk, alpha=0.75,
                    plan=xt.make_plan(XB.METHOD_FUSED, moduli=moduli))
    assert st.moduli == moduli and st.products == moduli
    assert err <= 2.0 ** (5 - st.residue_bits), (moduli, st.residue_bits, err)
    if moduli >= 14:
        assert err <= TOL[dtk], err


def test_residues_and_slices_agree(xt, dev):
    """Both FP64 schemes on the same contraction: within their bounds of each other."""
    ext = {"a": 24, "b": 20, "c": 16, "d": 12, "i": 10, "j": 9}
    pat = "D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)"
    e1, s1 = fused(xt, dev, pat, ext, O.R8, plan=xt.make_plan(XB.METHOD_FUSED), seed=9)
    e2, s2 = fused(xt, dev, pat, ext, O.R8, plan=xt.make_plan(XB.METHOD_FUSED, slices=6), seed=9)
    assert s1.moduli > 0 and s2.moduli == 0
    assert e1 <= TOL[O.R8] and e2 <= TOL[O.R8]


@pytest.mark.parametrize("dtk", [O.R8, O.R4, O.C8, O.C4])
def test_fused_padded_shapes(xt, dev, dtk):
    err, _ = fused(xt, dev, "D(i,j)+=L(k,i)*R(k,j)", {"i": 130, "j": 70, "k": 200}, dtk, alpha=0.75)
    assert err <= TOL[dtk], err


@pytest.mark.parametrize("dtk", [O.R8, O.R4, O.C8, O.C4])
@pytest.mark.parametrize("pattern,ext", [
    ("D(a,b,c,d)+=L(c,k,a,l)*R(l,d,k,b)", {"a": 12, "b": 11, "c": 13, "d": 10, "k": 9, "l": 14}),
    ("D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)", {"a": 16, "b": 16, "c": 16, "d": 16, "i": 8, "j": 8}),
    ("D(a,i,b,j)+=L(a,k,c,i)*R(c,b,k,j)", {"a": 16, "b": 16, "c": 16, "i": 8, "j": 8, "k": 8}),
    ("D(j,i)+=L(i,k)*R(j,k)", {"i": 300, "j": 200, "k": 128}),
])
def test_fused_tensor_patterns(xt, dev, dtk, pattern, ext):
    for accumulative, alpha in ((True, 0.5), (False, -1.25 + (0.5j if dtk in (O.C4, O.C8) else 0))):
        err, _ = fused(xt, dev, pattern, ext, dtk, alpha, accumulative)
        assert err <= TOL[dtk], (pattern, accumulative, err)


@pytest.mark.parametrize("dtk", [O.C8, O.C4])
@pytest.mark.parametrize("pattern", ["D(a,b)+=L+(k,a)*R(k,b)", "D(a,b)+=L(k,a)*R+(k,b)", "D+(a,b)+=L(k,a)*R(k,b)"])
def test_fused_conjugation(xt, dev, dtk, pattern):
    err, _ = fused(xt, dev, pattern, {"a": 150, "b": 90, "k": 170}, dtk, alpha=0.7 - 0.2j)
    assert err <= TOL[dtk], err


@pytest.mark.parametrize("slices,bound", [(4, 1e-7), (5, 1e-9), (6, 1e-12), (7, 1e-13)])
def test_slice_count_accuracy(xt, dev, slices, bound):
    """Fewer slices trade accuracy for speed; every count stays within its bound."""
    err, st = fused(xt, dev, "D(i,j)+=L(k,i)*R(k,j)", {"i": 256, "j": 192, "k": 320}, O.R8,
                    plan=xt.make_plan(XB.METHOD_FUSED, slices=slices))
    assert st.slices == slices
    assert err <= bound, err


def test_bf16_three_and_four_terms(xt, dev):
    """The hi*lo cross terms carry the accuracy; the lo*lo term adds nothing
    measurable because the two-part split itself keeps ~16 mantissa bits."""
    e3, _ = fused(xt, dev, "D(i,j)+=L(k,i)*R(k,j)", {"i": 256, "j": 256, "k": 512}, O.R4,
                  plan=xt.make_plan(XB.METHOD_FUSED, bf16_terms=3))
    e4, _ = fused(xt, dev, "D(i,j)+=L(k,i)*R(k,j)", {"i": 256, "j": 256, "k": 512}, O.R4,
                  plan=xt.make_plan(XB.METHOD_FUSED, bf16_terms=4))
    assert e3 <= 1e-4 and e4 <= 1e-4
    assert e4 <= 1.2 * e3


def test_tile_n_128_and_256_agree(xt, dev):
    ext = {"i": 256, "j": 512, "k": 256}
    e1, _ = fused(xt, dev, "D(i,j)+=L(k,i)*R(k,j)", ext, O.R8, plan=xt.make_plan(XB.METHOD_FUSED, tile_n=128))
    e2, _ = fused(xt, dev, "D(i,j)+=L(k,i)*R(k,j)", ext, O.R8, plan=xt.make_plan(XB.METHOD_FUSED, tile_n=256))
    assert e1 <= TOL[O.R8] and e2 <= TOL[O.R8]


def test_kat_single_block_40(xt, dev):
    """The 40^4 single-block contraction with constant inputs (closed form)."""
    pattern = "D(a,b,c,d)+=L(c,k,a,l)*R(l,d,k,b)"
    dims = [40] * 4
    d = np.zeros(40 ** 4); l = np.full(40 ** 4, 0.01); r = np.full(40 ** 4, 0.001)
    got = run_gpu(xt, dev, pattern, d, dims, l, dims, r, dims, 0.5, True, XB.METHOD_FUSED)
    assert np.allclose(got, 1600 * 0.01 * 0.001 * 0.5, rtol=1e-12, atol=0)


def test_long_k_splits_exact_int32_passes(xt, dev):
    """K = 131200 (1025 K blocks) with every slice below the top equal to -128:
    each K block adds exactly 2^21 to an INT32 accumulator, so a pass may hold at
    most 1023 blocks.  The slice pairs (INT8 slices, on request) must be split
    along K into exact passes, and the residue products (the default) into K
    chunks whose residues add up mod m; an overflow would show as a grossly
    wrong D."""
    from fractions import Fraction
    K, M, N = 131200, 128, 64
    word = 63 * 2 ** 48 + 128 * sum(2 ** (8 * i) for i in range(6))
    v = -word / 2.0 ** 55                      # balanced digits (-63, -128, ..., -128)
    assert Fraction(v) == Fraction(-word, 2 ** 55)
    l = np.full(K * M, v); r = np.full(K * N, v)
    want = float(Fraction(v) ** 2 * K / 2)
    pat = "D(i,j)+=L(k,i)*R(k,j)"
    for plan in (xt.make_plan(XB.METHOD_FUSED, moduli=-1), xt.make_plan(XB.METHOD_FUSED)):
        dd, ld, rd = dev.put(np.zeros(M * N)), dev.put(l), dev.put(r)
        xt.tensor_contract(pat, O.R8, [M, N], dd.data_ptr(), [K, M], ld.data_ptr(), [K, N], rd.data_ptr(), 0.5,
                           accumulative=True, plan=plan, stream=dev.stream())
        got = dev.get(dd, np.float64, M * N)
        st = xt.last_contract_stats()
        assert st.method == XB.METHOD_FUSED
        if st.moduli:
            assert st.products == st.moduli and st.passes == 2 * st.moduli
        else:
            assert st.products == 21 and st.passes > 6
        assert np.allclose(got, want, rtol=1e-13, atol=0), (st.moduli, got[:4], want)


@pytest.mark.parametrize("dtk", [O.R8, O.C8, O.R4, O.C4])
def test_sm_pair_and_single_sm_tiles_agree(xt, dev, dtk):
    """The CTA-pair kernel (256-row tiles over two SMs) and the single-SM
    kernel (128-row tiles) compute the same sums; for the INT8 slices every
    partial sum is exact, so R8/C8 results agree bit for bit."""
    pattern, ext = "D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)", {"a": 24, "b": 20, "c": 16, "d": 12, "i": 10, "j": 9}
    errs, outs = [], []
    for tm in (128, 256):
        err, st = fused(xt, dev, pattern, ext, dtk, alpha=0.5, plan=xt.make_plan(XB.METHOD_FUSED, tile_m=tm), seed=5)
        errs.append(err)
    assert max(errs) <= TOL[dtk], errs
    if dtk in (O.R8, O.C8):
        ddims, ldims, rdims = shapes(pattern, ext)
        vol = lambda s: int(np.prod(s))
        d, l, r = rand_host(dtk, vol(ddims), 5), rand_host(dtk, vol(ldims), 6), rand_host(dtk, vol(rdims), 7)
        for tm in (128, 256):
            dd, ld, rd = dev.put(d), dev.put(l), dev.put(r)
            xt.tensor_contract(pattern, dtk, ddims, dd.data_ptr(), ldims, ld.data_ptr(), rdims, rd.data_ptr(), 0.5,
                               plan=xt.make_plan(XB.METHOD_FUSED, tile_m=tm), stream=dev.stream())
            outs.append(dev.get(dd, d.dtype, d.size))
        assert np.array_equal(outs[0].view(np.uint8), outs[1].view(np.uint8))
