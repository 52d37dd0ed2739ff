"""GPU checks of the block-sparse caller side: task lists produced from segment
metadata (tb_bsc_tasks_from_blocks) and block contractions batched by the
caller (tb_batch_*), against the per-block loop of plain contractions that
the reference's TAVP-WRK issues (one talsh_tensor_contract per block,
INTERVIRT/tavp_worker.F90:9467)."""
import numpy as np
import pytest

import exatensor_b200 as XB
import oracle as O
from exatensor_b200 import blocksparse as BS
from tests.test_gpu_bsc import PATTERN, make_problem, per_block_loop, values

pytestmark = pytest.mark.gpu
TOL = {O.R8: 1e-12, O.R4: 1e-4, O.C8: 1e-12}


def segment_lists(T):
    keys = list(T.blocks)
    return T.segments, keys, [T.ptr(k) for k in keys]


@pytest.mark.parametrize("dtk", [O.R8, O.R4])
def test_batch_of_produced_tasks_matches_per_block_loop(xt, dev, dtk):
    import torch
    L, R, D, tasks_py, _ = make_problem(xt, dev, dtk, seed=21)
    tasks = XB.bsc_tasks_from_blocks(PATTERN, segment_lists(D), segment_lists(L), segment_lists(R))
    assert sorted(tasks) == sorted(tasks_py)
    ref = per_block_loop(xt, dev, dtk, D, tasks, 0.5, False)
    b = XB.Batch(PATTERN, dtk, alpha=0.5, accumulative=False)
    for i in range(0, len(tasks), 7):  # the caller adds its block instructions as they come
        b.add(tasks[i:i + 7])
    assert b.pending() == len(tasks)
    b.flush(stream=dev.stream())
    torch.cuda.synchronize()
    xt.device_check(dev.stream())
    dt = O.NP_DTYPE[dtk]
    assert O.rel_frobenius(values(D, D.data, dt), values(D, ref, dt)) <= TOL[dtk]
    first = D.data.clone()
    # the same list again: the cached plan runs (timed once on this second use)
    b.add(tasks)
    b.flush(stream=dev.stream())
    torch.cuda.synchronize()
    assert O.rel_frobenius(values(D, D.data, dt), values(D, first, dt)) <= TOL[dtk]
    st = b.stats()
    assert (st.plans_built, st.plan_reuses, st.autotunes, st.grouped_flushes, st.cached_plans) == (1, 1, 1, 2, 1)
    assert st.tasks == 2 * len(tasks) and b.pending() == 0
    b.close()


def test_batch_accumulates_each_output_block_once_per_flush(xt, dev):
    import torch
    L, R, D, tasks, _ = make_problem(xt, dev, O.R8, seed=22)
    d0 = D.data.clone()
    ref = per_block_loop(xt, dev, O.R8, D, tasks, 1.0, True)
    b = XB.Batch(PATTERN, O.R8, accumulative=True)
    b.add(tasks)
    b.flush(stream=dev.stream())
    torch.cuda.synchronize()
    dt = np.float64
    assert O.rel_frobenius(values(D, D.data, dt), values(D, ref, dt)) <= 1e-12
    assert not torch.equal(d0, D.data)
    b.close()


def test_complex_batch_runs_as_a_loop(xt, dev):
    import torch
    rng = np.random.default_rng(5)
    es = 16
    segs = BS.random_segments(4, 2, 6, 12, rng)
    segr = [segs[2], segs[3]] + BS.random_segments(2, 2, 6, 12, rng)
    L = BS.BlockSparseTensor(segs, BS.random_keys(segs, 0.6, rng), es)
    R = BS.BlockSparseTensor(segr, BS.random_keys(segr, 0.6, rng), es)
    xt.fill_uniform(O.C8, L.volume, L.data.data_ptr(), 1, stream=dev.stream())
    xt.fill_uniform(O.C8, R.volume, R.data.data_ptr(), 2, stream=dev.stream())
    D, tasks, _ = BS.contraction_tasks(PATTERN, L, R)
    xt.fill_uniform(O.C8, D.volume, D.data.data_ptr(), 3, stream=dev.stream())
    ref = per_block_loop(xt, dev, O.C8, D, tasks, 1.0, False)
    b = XB.Batch(PATTERN, O.C8, accumulative=False)
    b.add(tasks)
    b.flush(stream=dev.stream())
    torch.cuda.synchronize()
    st = b.stats()
    assert st.loop_flushes == 1 and st.grouped_flushes == 0
    assert O.rel_frobenius(values(D, D.data, np.complex128), values(D, ref, np.complex128)) <= 1e-12
    b.close()


def test_batch_rejects_bad_requests(xt):
    with pytest.raises(XB.TBError):
        XB.Batch("D(a)+=L(a)", O.R8)      # not a contraction
    with pytest.raises(XB.TBError):
        XB.Batch(PATTERN, 3)              # not a data kind
