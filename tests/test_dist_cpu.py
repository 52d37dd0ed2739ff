"""Multi-process plumbing of bench.py on CPU: two ranks over gloo (the GPU
runs use NCCL with the same calls).  The path has no collective in its data
flow -- ranks run independent replicas -- so what needs checking is the
rendezvous, the barrier and the max-over-ranks timing reduction."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "BENCH_DIST_BACKEND": "gloo"})
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_setup(world)
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(w)
    t = bench.max_over_ranks(10.0 + 5.0 * rank, w)     # per-rank "times"
    out[rank] = t
    bench.barrier(w)
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_barrier_and_max_over_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert dict(out) == {0: 15.0, 1: 15.0}  # every rank sees the slowest rank's time


def _ref_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "BENCH_DIST_BACKEND": "gloo"})
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import argparse

    import bench
    calls = []
    bench.cpu_contraction_sample = lambda steps=1, **kw: calls.append(steps) or None  # no CPU work in this test
    bench.run_reference(argparse.Namespace(gpus=world, steps=1, warmup=0, workload="ccsd1_r8"))
    out[rank] = len(calls)


@pytest.mark.timeout(120)
def test_reference_arm_runs_on_rank_zero_only():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_ref_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert dict(out) == {0: 1, 1: 0}
