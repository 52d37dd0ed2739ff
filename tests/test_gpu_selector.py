"""GPU checks of the learned plan selector: the network's CUDA forward and
backward kernels against the NumPy reference (values and gradients), that
training with them fits, and that the trained selector, used by METHOD_AUTO,
beats the size rule on held-out timings of the recorded corpus."""
import os

import numpy as np
import pytest

import exatensor_b200 as XB
import oracle as O
from exatensor_b200 import selector as S
from tests import mlp_ref

pytestmark = pytest.mark.gpu
CORPUS = os.path.join(os.path.dirname(__file__), "golden", "selector_corpus.npz")


def _net(nin=16, nh=64, nout=3, batch=96, seed=3):
    return XB.MLP(nin, nh, nout, max_batch=batch, seed=seed)


def test_forward_matches_reference(xt):
    import torch
    rng = np.random.default_rng(1)
    net = _net()
    p = net.params()
    x = rng.normal(0, 1, (80, 16)).astype(np.float32)
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty((80, 3), dtype=torch.float32, device="cuda")
    net.forward(dx.data_ptr(), 80, dy.data_ptr())
    torch.cuda.synchronize()
    ref, _ = mlp_ref.forward(p, x.astype(np.float64), 16, 64, 3)
    assert np.allclose(dy.cpu().numpy(), ref, rtol=1e-4, atol=1e-5)
    net.close()


def test_gradients_match_reference_and_finite_differences(xt):
    import torch
    rng = np.random.default_rng(2)
    net = _net()
    p = net.params()
    x = rng.normal(0, 1, (96, 16)).astype(np.float32)
    t = rng.normal(0, 1, (96, 3)).astype(np.float32)
    t[::7, 1] = np.nan  # unlabelled entries
    dx, dt = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    loss = net.backward(dx.data_ptr(), dt.data_ptr(), 96)
    g = net.params(grads=True)
    ref_loss, ref_g = mlp_ref.loss_and_grad(p, x, t, 16, 64, 3)
    assert np.isclose(loss, ref_loss, rtol=1e-4)
    assert np.allclose(g, ref_g, rtol=2e-3, atol=2e-6 * np.abs(ref_g).max())
    # central differences on a few parameters of each layer (float64 reference)
    for k in (0, 16 * 64 + 5, 16 * 64 + 64 + 300, len(p) - 2):
        h = 1e-4
        pp, pm = p.astype(np.float64).copy(), p.astype(np.float64).copy()
        pp[k] += h
        pm[k] -= h
        fd = (mlp_ref.loss_and_grad(pp, x, t, 16, 64, 3)[0] - mlp_ref.loss_and_grad(pm, x, t, 16, 64, 3)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-3 * max(1.0, abs(fd)), (k, fd, g[k])
    net.close()


def test_training_fits_a_smooth_target(xt):
    rng = np.random.default_rng(4)
    X = rng.normal(0, 1, (2048, 16)).astype(np.float32)
    Y = np.stack([np.sin(X[:, 0]) + X[:, 1] ** 2 / 4, X[:, 2] * X[:, 3] / 2, np.abs(X[:, 4])], 1).astype(np.float32)
    params, mean, scale, hist = S.train(X, Y, hidden=64, epochs=60, batch=256, lr=3e-3, seed=0, log_every=10)
    assert hist[-1][1] < 0.2 * hist[0][1], hist
    pred = S.predict(params, mean, scale, X, hidden=64)
    assert np.mean((pred - Y) ** 2) < 0.1


@pytest.mark.skipif(not os.path.exists(CORPUS), reason="recorded selector corpus not present")
def test_trained_selector_beats_the_size_rule(xt):
    d = np.load(CORPUS)
    F, T = d["features"], d["log_ms"]
    assert T.shape[1] == XB.SELECT_PLANS == len(S.PLANS)
    always = [i for i in range(T.shape[1]) if i not in S.FP64_ONLY]
    ok = np.isfinite(T[:, always]).all(axis=1)
    n_train = int(ok[:int(0.8 * len(F))].sum())  # the first 80% of the entries train
    F, T = F[ok], T[ok]
    params, mean, scale, _ = S.train(F[:n_train], T[:n_train], hidden=128, epochs=150, seed=0)
    pred = S.predict(params, mean, scale, F[n_train:], hidden=128)
    learned = S.evaluate(T[n_train:], S.choose(pred, F[n_train:]))
    rule = S.evaluate(T[n_train:], [S.rule_choice(f) for f in F[n_train:]])
    assert learned["total_time_regret"] < rule["total_time_regret"], (learned, rule)
    assert learned["mean_regret"] < rule["mean_regret"], (learned, rule)


def test_auto_uses_the_installed_selector(xt, dev):
    """With a selector installed, METHOD_AUTO runs the plan it predicts fastest,
    and the result stays within that plan's tolerance; with the autotune
    fallback forced, every candidate is timed once and D is unchanged by it."""
    from tests.test_gpu_contract import oracle_dd, shapes
    from tests.test_gpu_permute import rand_host
    pattern, ext = "D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)", {"a": 24, "b": 20, "c": 16, "d": 12, "i": 10, "j": 9}
    ddims, ldims, rdims = shapes(pattern, ext)
    vol = lambda s: int(np.prod(s))
    d, l, r = rand_host(O.R8, vol(ddims), 1), rand_host(O.R8, vol(ldims), 2), rand_host(O.R8, vol(rdims), 3)
    exact = oracle_dd(pattern, d, ddims, l, ldims, r, rdims, 1.0, True)
    nh, P = 8, XB.SELECT_PLANS
    n = 16 * nh + nh + nh * nh + nh + nh * P + P
    for favoured, method in ((0, XB.METHOD_TTGT), (2, XB.METHOD_FUSED)):
        p = np.zeros(n, np.float32)
        p[-P:] = 5.0
        p[-P + favoured] = 1.0           # constant prediction: this plan is fastest
        XB.selector_install(nh, p, np.zeros(16, np.float32), np.ones(16, np.float32))
        try:
            dd, ld, rd = dev.put(d), dev.put(l), dev.put(r)
            xt.tensor_contract(pattern, O.R8, ddims, dd.data_ptr(), ldims, ld.data_ptr(), rdims, rd.data_ptr(),
                               1.0, stream=dev.stream())
            got = dev.get(dd, np.float64, d.size)
            assert xt.last_contract_stats().method == method
            assert O.rel_frobenius(got, exact) <= 1e-12
        finally:
            XB.selector_install(0, None, None, None)
    # autotune fallback (large contractions only): equal predictions are
    # ambiguous for any margin > 0, so every candidate is timed once with
    # alpha = 0, beta = 1; D must come out as one plain contraction would make it
    pattern2, m = "D(i,j)+=L(k,i)*R(k,j)", 2048
    d2, l2, r2 = rand_host(O.R8, m * m, 4), rand_host(O.R8, m * m, 5), rand_host(O.R8, m * m, 6)
    dd, ld, rd = dev.put(d2), dev.put(l2), dev.put(r2)
    xt.tensor_contract(pattern2, O.R8, [m, m], dd.data_ptr(), [m, m], ld.data_ptr(), [m, m], rd.data_ptr(), 1.0,
                       plan=xt.make_plan(XB.METHOD_TTGT), stream=dev.stream())
    want = dev.get(dd, np.float64, d2.size)
    XB.selector_install(nh, np.zeros(n, np.float32), np.zeros(16, np.float32), np.ones(16, np.float32),
                        margin=0.5, autotune=True)
    try:
        for _ in range(3):  # first: prediction; second: timed candidates; third: cached decision
            dd = dev.put(d2)
            xt.tensor_contract(pattern2, O.R8, [m, m], dd.data_ptr(), [m, m], ld.data_ptr(), [m, m], rd.data_ptr(),
                               1.0, stream=dev.stream())
            got = dev.get(dd, np.float64, d2.size)
            assert xt.last_contract_stats().method in (XB.METHOD_TTGT, XB.METHOD_FUSED)
            assert O.rel_frobenius(got, want) <= 1e-12
    finally:
        XB.selector_install(0, None, None, None)
    xt.device_check(dev.stream())


def test_close_predictions_time_only_the_close_plans(xt, dev):
    """A large contraction whose network predictions put the 256-wide tile on
    one SM and on an SM pair within the margin of each other, and every other
    plan far behind, is timed on its second call on those two plans only.
    Whichever tile is kept, the residue products are exact, so D equals the
    single-SM plan's result bit for bit."""
    from tests.test_gpu_permute import rand_host
    m = 3328  # 2 * m^3 = 7.4e10 FLOP
    pattern = "D(i,j)+=L(k,i)*R(k,j)"
    d, l, r = rand_host(O.R8, m * m, 7), rand_host(O.R8, m * m, 8), rand_host(O.R8, m * m, 9)
    ld, rd = dev.put(l), dev.put(r)
    dd = dev.put(d)
    xt.tensor_contract(pattern, O.R8, [m, m], dd.data_ptr(), [m, m], ld.data_ptr(), [m, m], rd.data_ptr(), 1.0,
                       plan=xt.make_plan(XB.METHOD_FUSED, tile_n=256), stream=dev.stream())
    want = dev.get(dd, np.float64, d.size)
    nh, P = 8, XB.SELECT_PLANS
    n = 16 * nh + nh + nh * nh + nh + nh * P + P
    p = np.zeros(n, np.float32)
    p[-P:] = 5.0
    p[-P + 2] = 1.0  # the 256-wide tile on one SM ...
    p[-P + 3] = 1.1  # ... and on an SM pair, within the margin
    XB.selector_install(nh, p, np.zeros(16, np.float32), np.ones(16, np.float32), margin=0.25, autotune=True)
    try:
        tiles = []
        for _ in range(3):  # first: prediction; second: the two close plans timed; third: kept choice
            dd = dev.put(d)
            xt.tensor_contract(pattern, O.R8, [m, m], dd.data_ptr(), [m, m], ld.data_ptr(), [m, m], rd.data_ptr(),
                               1.0, stream=dev.stream())
            got = dev.get(dd, np.float64, d.size)
            st = xt.last_contract_stats()
            assert st.method == XB.METHOD_FUSED and st.tile_n == 256 and st.moduli > 0
            tiles.append(st.tile_m)
            assert np.array_equal(got.view(np.uint8), want.view(np.uint8))
        assert tiles[0] == 128 and tiles[1] == tiles[2] and tiles[2] in (128, 256)
    finally:
        XB.selector_install(0, None, None, None)
    xt.device_check(dev.stream())


def test_fp64_only_plan_is_never_chosen_for_fp32(xt):
    """The INT8-slice plan applies to FP64 data only: for an FP32 descriptor
    the selector passes over it even when it is predicted fastest."""
    nh, P = 8, XB.SELECT_PLANS
    n = 16 * nh + nh + nh * nh + nh + nh * P + P
    p = np.zeros(n, np.float32)
    p[-P:] = 5.0
    p[-P + 4] = 0.5  # slices predicted fastest
    p[-P + 1] = 1.0
    XB.selector_install(nh, p, np.zeros(16, np.float32), np.ones(16, np.float32))
    try:
        f64 = XB.contract_descriptor("D(i,j)+=L(k,i)*R(k,j)", 8, [512, 512], [512, 512], [512, 512])
        f32 = XB.contract_descriptor("D(i,j)+=L(k,i)*R(k,j)", 4, [512, 512], [512, 512], [512, 512])
        assert XB.selector_choose(f64)[0] == 4
        assert XB.selector_choose(f32)[0] == 1
        assert XB.selector_time(f64, 1000) > 0
    finally:
        XB.selector_install(0, None, None, None)
