"""CPU checks of the bench's workload definitions and of its independent
on-device checkers: the permutation sweep's shapes hold the governing
256 MiB volume, torch's permute (as the bench orders it) gives the oracle's
bits for every O2N permutation, and torch's d + l * scale gives the oracle's
two-rounding add bits (the bench compares every timed sweep case with these)."""
import itertools

import numpy as np
import pytest
import torch

import bench
import oracle as O
from tests.test_gpu_permute import rand_host


def test_sweep_shapes_and_classes():
    cases = bench.sweep_cases()
    classes = {c["cls"] for c in cases}
    for tag in ("r8", "r4"):
        for rank in range(2, 7):
            assert f"{tag}_{rank}" in classes
        for rank in (3, 4, 6):
            assert f"{tag}_{rank}s" in classes
    for c in cases:
        nbytes = bench.vol(c["dims"]) * (8 if c["dtk"] == 8 else 4)
        assert 0.9 * 2 ** 28 <= nbytes <= 1.1 * 2 ** 28, c
        assert sorted(c["perm"]) == list(range(1, len(c["dims"]) + 1))
        if c["cls"].endswith("s"):
            assert min(c["dims"]) <= 7
    assert sum(c["cls"] == "r8_4" for c in cases) == 24
    assert sum(c["cls"] == "r4_6" for c in cases) == 40
    assert len({c["perm"] for c in cases if c["cls"] == "r8_6"}) == 40
    assert len(bench.add_cases()) == 68


@pytest.mark.parametrize("dims", [[3, 4], [3, 4, 5], [2, 3, 4, 5], [2, 3, 1, 4, 2], [2, 3, 2, 3, 2, 2]])
def test_torch_permute_order_matches_oracle(dims):
    x = rand_host(O.R8, int(np.prod(dims)), 3)
    t = torch.from_numpy(x.copy()).view(torch.uint8)
    for perm in itertools.permutations(range(1, len(dims) + 1)):
        got = bench.torch_permuted(t, dims, perm, torch.int64).numpy().view(np.float64)
        assert np.array_equal(got, O.permute(x, dims, list(perm))), perm


@pytest.mark.parametrize("dtk", [O.R4, O.R8])
def test_torch_add_matches_oracle_bits(dtk):
    dims = [6, 5, 4, 3]
    n = int(np.prod(dims))
    l, d0 = rand_host(dtk, n, 8), rand_host(dtk, n, 9)
    fdt = torch.float64 if dtk == O.R8 else torch.float32
    for perm in [(1, 2, 3, 4), (3, 1, 4, 2), (4, 3, 2, 1)]:
        ref = O.tensor_add(list(perm), d0.copy(), l, dims, 0.37)
        lt = torch.from_numpy(l.copy()).view(torch.uint8)
        got = torch.from_numpy(d0.copy()) + bench.torch_permuted(lt, dims, perm, fdt) * 0.37
        assert np.array_equal(got.numpy().view(np.uint8), ref.view(np.uint8)), perm


def test_cpu_sample_shapes():
    """The CPU legs' sample: the headline pattern with a cut to 48 (1/4 of the
    v=192 FLOPs), N and K unchanged."""
    wl = bench.WORKLOADS["ccsd1_r8"]
    dd, ld, rd = bench.shapes(wl["pattern"], wl["v"], wl["o"])
    full = 2.0 * bench.vol(dd) * (bench.vol(ld) * bench.vol(rd) / bench.vol(dd)) ** 0.5
    dd[0], ld[0] = bench.CPU_SAMPLE_A, bench.CPU_SAMPLE_A
    part = 2.0 * bench.vol(dd) * (bench.vol(ld) * bench.vol(rd) / bench.vol(dd)) ** 0.5
    assert abs(part / full - 0.25) < 1e-12


def test_seeded_fill_matches_generator():
    a = O.fill_uniform(100003, 11)
    assert np.array_equal(a, O.splitmix64_uniform(100003, 11))
