"""GPU checks of block-sparse contractions run as one grouped launch
(tb_bsc_*), against the per-block loop of plain contractions that the
reference's hierarchical layer issues (one talsh_tensor_contract per block)."""
import numpy as np
import pytest

import exatensor_b200 as XB
import oracle as O
from exatensor_b200 import blocksparse as BS

pytestmark = pytest.mark.gpu
PATTERN = "D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)"


def make_problem(xt, dev, dtk, nseg=3, lo=8, hi=24, presence=0.5, seed=7):
    rng = np.random.default_rng(seed)
    es = xt.ELEM_BYTES[dtk]
    segs = BS.random_segments(4, nseg, lo, hi, rng)   # a, b, c, d of L
    segr = [segs[2], segs[3]] + BS.random_segments(2, nseg, lo, hi, rng)  # c, d, i, j of R
    L = BS.BlockSparseTensor(segs, BS.random_keys(segs, presence, rng), es)
    R = BS.BlockSparseTensor(segr, BS.random_keys(segr, presence, rng), es)
    xt.fill_uniform(dtk, L.volume, L.data.data_ptr(), seed + 1, stream=dev.stream())
    xt.fill_uniform(dtk, R.volume, R.data.data_ptr(), seed + 2, stream=dev.stream())
    D, tasks, pairs = BS.contraction_tasks(PATTERN, L, R)
    xt.fill_uniform(dtk, D.volume, D.data.data_ptr(), seed + 3, stream=dev.stream())
    return L, R, D, tasks, pairs


def per_block_loop(xt, dev, dtk, D, tasks, alpha, accumulative, method=XB.METHOD_TTGT):
    """The reference's scheme: one plain contraction per block task."""
    import torch
    out = D.data.clone()
    base = D.data.data_ptr()
    if not accumulative:
        for key, (off, dims) in D.blocks.items():
            n = int(np.prod(dims)) * D.elem_bytes
            out[off * D.elem_bytes: off * D.elem_bytes + n].zero_()
    for dp, dd, lp, ld, rp, rd in tasks:
        xt.tensor_contract(PATTERN, dtk, dd, out.data_ptr() + (dp - base), ld, lp, rd, rp, alpha,
                           accumulative=True, plan=xt.make_plan(method), stream=dev.stream())
    torch.cuda.synchronize()
    return out


def values(D, buf, dtype):
    a = buf.cpu().numpy().view(dtype)
    parts = [a[off: off + int(np.prod(dims))] for off, dims in D.blocks.values()]
    return np.concatenate(parts)


@pytest.mark.parametrize("dtk,tol", [(O.R8, 1e-12), (O.R4, 1e-4)])
@pytest.mark.parametrize("accumulative,alpha", [(True, 1.0), (False, 0.5)])
def test_grouped_matches_per_block_loop(xt, dev, dtk, tol, accumulative, alpha):
    import torch
    L, R, D, tasks, pairs = make_problem(xt, dev, dtk)
    assert len(tasks) > len(D.blocks)  # some output blocks receive several products
    ref = per_block_loop(xt, dev, dtk, D, tasks, alpha, accumulative)
    plan = XB.BlockSparsePlan(PATTERN, dtk, tasks, alpha=alpha, accumulative=accumulative, stream=dev.stream())
    plan.execute(stream=dev.stream())
    torch.cuda.synchronize()
    xt.device_check(dev.stream())
    dt = O.NP_DTYPE[dtk]
    got, want = values(D, D.data, dt), values(D, ref, dt)
    assert O.rel_frobenius(got, want) <= tol
    inf = plan.info()
    assert inf.tasks == len(tasks) and inf.out_blocks == len(D.blocks)
    plan.close()


def test_graph_replay_is_deterministic(xt, dev):
    import torch
    L, R, D, tasks, _ = make_problem(xt, dev, O.R8, seed=11)
    plan = XB.BlockSparsePlan(PATTERN, O.R8, tasks, accumulative=False, stream=dev.stream())
    plan.execute(stream=dev.stream())
    first = D.data.clone()
    plan.execute(stream=dev.stream())
    torch.cuda.synchronize()
    assert torch.equal(first, D.data)
    plan.execute(stream=dev.stream(), graph=False)
    torch.cuda.synchronize()
    assert torch.equal(first, D.data)
    plan.close()


def test_autotune_leaves_output_and_keeps_accuracy(xt, dev):
    import torch
    L, R, D, tasks, _ = make_problem(xt, dev, O.R8, seed=13)
    before = D.data.clone()
    plan = XB.BlockSparsePlan(PATTERN, O.R8, tasks, accumulative=True, stream=dev.stream())
    plan.autotune(stream=dev.stream())
    torch.cuda.synchronize()
    assert torch.equal(before, D.data)
    inf = plan.info()
    assert inf.tile_n in (128, 256) and inf.slices in (6, 7)
    assert inf.tune_ms[0] > 0 and inf.tune_ms[2] > 0
    ref = per_block_loop(xt, dev, O.R8, D, tasks, 1.0, True)
    plan.execute(stream=dev.stream())
    torch.cuda.synchronize()
    assert O.rel_frobenius(values(D, D.data, np.float64), values(D, ref, np.float64)) <= 1e-12
    plan.close()


def test_one_block_against_the_oracle(xt, dev):
    """One output block receiving several products, checked against the
    double-double oracle."""
    import torch
    L, R, D, tasks, pairs = make_problem(xt, dev, O.R8, nseg=2, presence=1.0, seed=17)
    key = next(iter(D.blocks))
    mine = [(t, p) for t, p in zip(tasks, pairs) if p[0] == key]
    assert len(mine) >= 2
    plan = XB.BlockSparsePlan(PATTERN, O.R8, [t for t, _ in mine], alpha=-0.75, accumulative=False,
                              stream=dev.stream())
    plan.execute(stream=dev.stream())
    torch.cuda.synchronize()
    off, dims = D.blocks[key]
    n = int(np.prod(dims))
    got = D.data.cpu().numpy().view(np.float64)[off: off + n]
    lv = L.data.cpu().numpy().view(np.float64)
    rv = R.data.cpu().numpy().view(np.float64)
    cptrn, *_ = O.parse_pattern(PATTERN)
    acc = np.zeros(n)
    for _, (_, lk, rk) in mine:
        lo, ldims = L.blocks[lk]
        ro, rdims = R.blocks[rk]
        O.contract(cptrn, acc, dims, lv[lo: lo + int(np.prod(ldims))].copy(), ldims,
                   rv[ro: ro + int(np.prod(rdims))].copy(), rdims, -0.75, 0, True, mode=1)
    assert O.rel_frobenius(got, acc) <= 1e-12
    plan.close()


def test_mismatched_block_is_rejected(xt, dev):
    L, R, D, tasks, _ = make_problem(xt, dev, O.R8, seed=19)
    dp, dd, lp, ld, rp, rd = tasks[0]
    bad = [(dp, dd, lp, ld, rp, rd), (dp, dd, lp, [x + 1 for x in ld], rp, rd)]
    with pytest.raises(XB.TBError):
        XB.BlockSparsePlan(PATTERN, O.R8, bad, stream=dev.stream())


def fixed_problem(xt, dev, dtk, segl, segr, seed):
    """Every block present, with the given segment extents (L: a b c d; R: c d i j)."""
    import itertools
    es = xt.ELEM_BYTES[dtk]
    L = BS.BlockSparseTensor(segl, list(itertools.product(*[range(len(s)) for s in segl])), es)
    R = BS.BlockSparseTensor(segr, list(itertools.product(*[range(len(s)) for s in segr])), es)
    xt.fill_uniform(dtk, L.volume, L.data.data_ptr(), seed + 1, stream=dev.stream())
    xt.fill_uniform(dtk, R.volume, R.data.data_ptr(), seed + 2, stream=dev.stream())
    D, tasks, pairs = BS.contraction_tasks(PATTERN, L, R)
    return L, R, D, tasks


@pytest.mark.parametrize("dtk,tol", [(O.R8, 1e-12), (O.R4, 1e-4)])
@pytest.mark.parametrize("tile_n", [128, 256])
def test_wide_blocks_and_long_block_sums(xt, dev, dtk, tol, tile_n):
    """Output blocks of many N tiles (items are issued N tile by N tile),
    and one output block whose pairs sum 1056 K blocks of INT8 planes
    (more than one exact INT32 pass holds, so passes end at pair
    boundaries), against the per-block loop of plain contractions."""
    import torch
    probs = [
        # 11 pairs of K = 96 * 128 into one 128 x 64 block
        ([[16], [8], [96] * 11, [128]], [[96] * 11, [128], [8], [8]]),
        # 256 x 3072 blocks: 24 (12) N tiles of 128 (256) columns
        ([[16], [16], [8], [8, 16]], [[8], [8, 16], [64], [48]]),
    ]
    for i, (segl, segr) in enumerate(probs):
        L, R, D, tasks = fixed_problem(xt, dev, dtk, segl, segr, 40 + i)
        ref = per_block_loop(xt, dev, dtk, D, tasks, 1.0, False)
        plan = XB.BlockSparsePlan(PATTERN, dtk, tasks, accumulative=False, plan=xt.make_plan(tile_n=tile_n),
                                  stream=dev.stream())
        plan.execute(stream=dev.stream())
        torch.cuda.synchronize()
        xt.device_check(dev.stream())
        assert plan.info().tile_n == tile_n
        dt = O.NP_DTYPE[dtk]
        assert O.rel_frobenius(values(D, D.data, dt), values(D, ref, dt)) <= tol, (i, tile_n)
        plan.close()
