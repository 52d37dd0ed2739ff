"""CPU check of the permutation kernel's index arithmetic.

Compiles tests/emul/perm_emul.cpp against the product's plan builder
(exatensor_b200/csrc/tb_perm_plan.cpp) and replays the tile kernel's load and
store loops for many shapes and permutations, asserting that every
shared-memory, table and global index stays in bounds and that each output
element is written exactly once with the right input element.
"""
import itertools
import os
import random
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def emul():
    d = tempfile.mkdtemp()
    exe = os.path.join(d, "perm_emul")
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", exe,
                    os.path.join(ROOT, "tests", "emul", "perm_emul.cpp"),
                    os.path.join(ROOT, "exatensor_b200", "csrc", "tb_perm_plan.cpp")], check=True)
    return exe


def run(exe, es, dims, perm, env=None):
    out = subprocess.run([exe, str(es), str(len(dims))] + [str(x) for x in dims] + [str(p) for p in perm],
                         capture_output=True, text=True, env=env)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("OK"), (dims, perm, out.stdout)


@pytest.mark.parametrize("es", [4, 8, 16])
def test_all_rank4_perms(emul, es):
    for perm in itertools.permutations([1, 2, 3, 4]):
        run(emul, es, [7, 5, 3, 9], perm)
        run(emul, es, [40, 40, 40, 40] if es != 16 else [20, 20, 20, 20], perm)


@pytest.mark.parametrize("es", [4, 8, 16])
def test_random_shapes(emul, es):
    rng = random.Random(1234 + es)
    for _ in range(150):
        rank = rng.randint(1, 6)
        dims = []
        for _ in range(rank):
            kind = rng.random()
            dims.append(rng.randint(1, 3) if kind < 0.25 else rng.randint(2, 7) if kind < 0.5
                        else rng.randint(8, 70))
        while True:
            vol = 1
            for x in dims:
                vol *= x
            if vol <= 400000:
                break
            i = max(range(rank), key=lambda k: dims[k])
            dims[i] = max(1, dims[i] // 2)
        perm = list(range(1, rank + 1))
        rng.shuffle(perm)
        run(emul, es, dims, perm)


def test_skewed_and_large_leading(emul):
    # one small extent, rest balanced; long preserved leading dimension
    run(emul, 8, [3, 200, 190], [3, 1, 2])
    run(emul, 8, [2, 90, 90, 9], [4, 3, 2, 1])
    run(emul, 4, [5000, 7, 3], [1, 3, 2])
    run(emul, 8, [4099, 5], [2, 1])
    run(emul, 16, [1, 33, 1, 17], [2, 4, 1, 3])
    run(emul, 8, [13, 5, 5, 16, 10, 5], [2, 5, 3, 4, 6, 1])  # store block inside the load block


@pytest.mark.parametrize("es", [4, 8])
def test_two_dimensional_vector_paths(emul, es):
    # shapes whose plans take the 2-D kernel's vector paths (column-group
    # transposes and row copies), with partial tiles at the edges
    for dims in ([90, 90, 30, 30], [90, 30, 90, 30], [66, 70, 18, 22], [100, 37, 45, 12], [38, 38, 38, 38]):
        for perm in ([1, 3, 2, 4], [2, 1, 3, 4], [2, 4, 1, 3], [1, 4, 3, 2], [3, 1, 2, 4], [4, 2, 3, 1]):
            run(emul, es, dims, perm)


@pytest.mark.parametrize("vmin,vmax,minrun", [(8, 24, 256), (24, 48, 256), (8, 16, 256), (4, 16, 128)])
def test_measured_choice_tile_bounds(emul, vmin, vmax, minrun):
    # the other tile-size bounds (and minimum runs) that large copies may be
    # timed with and run; the small ones are the list kernel's candidates
    env = dict(os.environ, TB_PERM_VMIN_KB=str(vmin), TB_PERM_VMAX_KB=str(vmax), TB_PERM_MINRUN=str(minrun))
    for es in (4, 8, 16):
        for perm in itertools.permutations([1, 2, 3, 4]):
            run(emul, es, [40, 40, 40, 40] if es != 16 else [20, 20, 20, 20], perm, env)
            run(emul, es, [7, 5, 3, 9], perm, env)
    for es in (4, 8):
        for dims in ([90, 90, 30, 30], [66, 70, 18, 22], [100, 37, 45, 12]):
            for perm in ([1, 3, 2, 4], [2, 1, 3, 4], [2, 4, 1, 3], [3, 4, 1, 2], [4, 3, 2, 1]):
                run(emul, es, dims, perm, env)
    rng = random.Random(77 + vmin + minrun)
    for _ in range(60):
        rank = rng.randint(2, 6)
        dims = [rng.randint(2, 40) for _ in range(rank)]
        while True:
            vol = 1
            for x in dims:
                vol *= x
            if vol <= 400000:
                break
            i = max(range(rank), key=lambda k: dims[k])
            dims[i] = max(1, dims[i] // 2)
        perm = list(range(1, rank + 1))
        rng.shuffle(perm)
        run(emul, rng.choice([4, 8, 16]), dims, perm, env)


@pytest.fixture(scope="module")
def plan_info():
    d = tempfile.mkdtemp()
    exe = os.path.join(d, "perm_plan_info")
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", exe,
                    os.path.join(ROOT, "tests", "emul", "perm_plan_info.cpp"),
                    os.path.join(ROOT, "exatensor_b200", "csrc", "tb_perm_plan.cpp")], check=True)
    return exe


@pytest.mark.parametrize("es,n", [(8, 76), (4, 90)])
def test_sweep_plans_take_the_fast_paths(plan_info, es, n):
    """The 24 rank-4 permutations of the 256 MiB sweep tensors plan onto the
    2-D kernel's fast paths: every plan is two-dimensional with full-tile
    offset lists (or the one-dimensional plain copy), no dimension split into
    a few tiles leaves a partial one, and store runs are at least 256 bytes."""
    for perm in itertools.permutations([1, 2, 3, 4]):
        out = subprocess.run([plan_info, str(es), "4"] + [str(n)] * 4 + [str(p) for p in perm],
                             capture_output=True, text=True, check=True).stdout.split()
        lin2d, vec2d, rows2d, lists, LB, pes, partial_small, ntiles = map(int, out)
        assert lin2d == 1, perm
        assert (vec2d or rows2d) and lists in (8, 16), (perm, out)
        assert partial_small == 0, (perm, out)
        assert LB * pes >= 256, (perm, out)


def test_offset_lists_decline_offsets_beyond_32_bits(plan_info):
    """The 2-D kernel's full-tile lists hold 32-bit offsets from a tile's
    origin.  For tensors whose tiles span more than 2^31 elements of output
    the planner must leave them off (the general code, with 64-bit offsets,
    runs); where the offsets fit, the lists stay on.  Planning only: no
    tensor of this size is allocated."""
    huge = [(8, [64, 1048576, 40], [3, 2, 1]), (8, [64, 67108864], [2, 1]),
            (4, [90, 90, 300000], [1, 3, 2]), (8, [76, 40000000, 76], [3, 2, 1])]
    for es, dims, perm in huge:
        out = subprocess.run([plan_info, str(es), str(len(dims))] + [str(x) for x in dims] + [str(p) for p in perm],
                             capture_output=True, text=True, check=True).stdout.split()
        lin2d, vec2d, rows2d, lists = map(int, out[:4])
        assert lin2d == 1 and (vec2d or rows2d) and lists == 0, (dims, perm, out)
    out = subprocess.run([plan_info, "8", "3", "76", "76", "1000000", "2", "1", "3"], capture_output=True, text=True,
                         check=True).stdout.split()
    assert int(out[3]) == 8, out


@pytest.mark.parametrize("minrun", [256, 128])
def test_sweep_shapes_general_plans(emul, minrun):
    """The permutation sweep's rank-5/6 and skewed shapes at reduced extents
    (the planner's structure, not the volume, decides the kernel), with the
    list kernel's small-tile candidates: lists, tables and partial tiles."""
    env = dict(os.environ, TB_PERM_VMIN_KB="4", TB_PERM_VMAX_KB="16", TB_PERM_MINRUN=str(minrun))
    rng = random.Random(5 + minrun)
    shapes = [[9, 9, 9, 9, 9], [6, 6, 6, 6, 6, 6], [5, 7, 6, 5, 6, 7], [3, 60, 60], [60, 60, 2], [5, 24, 24, 24],
              [24, 24, 24, 7], [2, 10, 10, 10, 10, 10], [10, 10, 10, 10, 10, 4]]
    for dims in shapes:
        for _ in range(6):
            perm = list(range(1, len(dims) + 1))
            rng.shuffle(perm)
            for es in (4, 8):
                run(emul, es, dims, perm, env)
