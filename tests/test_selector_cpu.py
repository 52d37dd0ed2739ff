"""Host-side parts of the learned plan selector: descriptors, the corpus
generator, regret arithmetic and the host inference used by METHOD_AUTO
(checked against the NumPy reference network)."""
import numpy as np
import pytest

import exatensor_b200 as XB
from exatensor_b200 import selector as S
from tests import mlp_ref


def test_descriptor_layout_flags():
    f = XB.contract_descriptor("D(i,j)+=L(k,i)*R(k,j)", 8, [30, 20], [40, 30], [40, 20])
    assert f.shape == (XB.DESC_FEATURES,)
    assert np.allclose(f[:3], np.log2([30, 20, 40]))
    assert f[12] == 1 and f[13] == 1 and f[14] == 1 and f[15] == 1
    g = XB.contract_descriptor("D(j,i)+=L(i,k)*R(j,k)", 4, [20, 30], [30, 40], [20, 40])
    assert g[12] == 0 and g[13] == 0 and g[14] == 0 and g[15] == 0
    assert np.isclose(g[3], np.log2(2.0 * 30 * 20 * 40))


def test_random_contractions_respect_the_corpus_limits():
    rng = np.random.default_rng(3)
    for _ in range(300):
        pattern, dd, ld, rd, dtk = S.random_contraction(rng)
        es = 8 if dtk == 8 else 4
        assert 2 <= len(ld) <= 6 and 2 <= len(rd) <= 6 and 1 <= len(dd) <= 6
        assert (np.prod(dd) + np.prod(ld) + np.prod(rd)) * es <= 4 << 30
        assert all(2 <= e <= 512 for e in dd + ld + rd)
        f = XB.contract_descriptor(pattern, dtk, dd, ld, rd)
        assert np.all(np.isfinite(f)) and 1 <= f[8] <= 4


def test_regret_arithmetic():
    t = np.array([[1.0, 2.0, 4.0], [3.0, 1.5, 1.0]])
    mean_r, total_r = S.regret(t, [0, 0])
    assert np.isclose(mean_r, (0 + 2.0) / 2) and np.isclose(total_r, 4.0 / 2.0 - 1.0)
    assert S.regret(t, [0, 2]) == (0.0, 0.0)


def test_host_inference_matches_the_reference_network():
    rng = np.random.default_rng(5)
    nh, P = 32, XB.SELECT_PLANS
    n = 16 * nh + nh + nh * nh + nh + nh * P + P
    p = rng.normal(0, 0.3, n).astype(np.float32)
    mean = rng.normal(0, 1, 16).astype(np.float32)
    scale = rng.uniform(0.5, 2, 16).astype(np.float32)
    XB.selector_install(nh, p, mean, scale)
    try:
        for _ in range(20):
            x = rng.normal(0, 3, 16).astype(np.float32)
            x[15] = 1.0  # an FP64 descriptor: every plan applies
            idx, y = XB.selector_choose(x)
            ref, _ = mlp_ref.forward(p, ((x - mean) / scale)[None, :], 16, nh, P)
            assert np.allclose(y, ref[0], rtol=1e-4, atol=1e-4)
            assert idx == int(np.argmin(y))
    finally:
        XB.selector_install(0, None, None, None)
    assert XB.selector_choose(np.zeros(16, np.float32))[0] == -1
