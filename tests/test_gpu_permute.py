"""GPU parity: permutations (tb_tensor_copy) are bit-exact against the oracle's
restatement of tensor_block_copy (TALSH/tensor_algebra_cpu.F90:3151,
:7699-7940), for every data kind, all 24 rank-4 permutations, random ranks 1-6
with unit, skewed and prime extents, complex conjugation, and at the full
256 MiB sweep size through inverse-permutation round trips."""
import itertools
import random

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
KINDS = [O.R4, O.R8, O.C4, O.C8]


def rand_host(dtk, vol, seed):
    x = O.splitmix64_uniform(vol * (2 if dtk in (O.C4, O.C8) else 1), seed)
    if dtk in (O.C4, O.C8):
        x = x[0::2] + 1j * x[1::2]
    return x.astype(O.NP_DTYPE[dtk])


def gpu_permute(xt, dev, x, dims, perm, conj_bits=0, scatter=False):
    dtk = O.DTK_OF[x.dtype]
    src = dev.put(x)
    dst = dev.empty(x.nbytes, fill=0xA5)
    xt.tensor_copy(dtk, dims, perm, src.data_ptr(), dst.data_ptr(), conj_bits, dev.stream(), scatter)
    return dev.get(dst, x.dtype, x.size)


@pytest.mark.parametrize("dtk", KINDS)
def test_all_rank4_permutations_bit_exact(xt, dev, dtk):
    dims = [5, 7, 3, 6]
    x = rand_host(dtk, int(np.prod(dims)), 11)
    for perm in itertools.permutations([1, 2, 3, 4]):
        ref = O.permute(x, dims, perm)
        got = gpu_permute(xt, dev, x, dims, perm)
        assert np.array_equal(got.view(np.uint8), ref.view(np.uint8)), perm
        got_s = gpu_permute(xt, dev, x, dims, perm, scatter=True)
        assert np.array_equal(got_s.view(np.uint8), ref.view(np.uint8)), perm


@pytest.mark.parametrize("dtk", KINDS)
def test_random_shapes_bit_exact(xt, dev, dtk):
    rng = random.Random(100 + dtk)
    for case in range(40):
        rank = rng.randint(1, 6)
        dims = [rng.choice([1, 2, 3, 5, 7, 13, 31, 40, 64, 97]) for _ in range(rank)]
        while np.prod(dims) > 300000:
            dims[int(np.argmax(dims))] //= 2
        perm = list(range(1, rank + 1))
        rng.shuffle(perm)
        x = rand_host(dtk, int(np.prod(dims)), case)
        ref = O.permute(x, dims, perm)
        got = gpu_permute(xt, dev, x, dims, perm)
        assert np.array_equal(got.view(np.uint8), ref.view(np.uint8)), (dims, perm)


@pytest.mark.parametrize("dtk", [O.C4, O.C8])
@pytest.mark.parametrize("conj_bits", [1, 2, 3])
def test_conjugating_copy(xt, dev, dtk, conj_bits):
    dims = [9, 4, 11]
    perm = [2, 3, 1]
    x = rand_host(dtk, int(np.prod(dims)), 3)
    lconj = bool((conj_bits & 1) ^ ((conj_bits >> 1) & 1))
    ref = O.permute(x, dims, perm, conj=lconj)
    got = gpu_permute(xt, dev, x, dims, perm, conj_bits)
    assert np.array_equal(got.view(np.uint8), ref.view(np.uint8))


def test_single_block_permutation_3142(xt, dev):
    """The 40^4 R8 permutation (3,1,4,2), read as O2N and as N2O."""
    dims = [40, 40, 40, 40]
    x = rand_host(O.R8, 40 ** 4, 0)
    for perm in ([3, 1, 4, 2], [2, 4, 1, 3]):
        ref = O.permute(x, dims, perm)
        assert np.array_equal(gpu_permute(xt, dev, x, dims, perm), ref)


# Shapes whose plans run the 2-D kernel's vector paths: column-group
# transposes (e.g. 2134) and row copies (1324, 1432: the fastest dim stays),
# with partial tiles at the edges (90 and 30 do not divide every tile).
TWO_D_SHAPES = [[90, 90, 30, 30], [90, 30, 90, 30], [66, 70, 18, 22], [100, 37, 45, 12], [38, 38, 38, 38]]
TWO_D_PERMS = [(1, 3, 2, 4), (2, 1, 3, 4), (2, 4, 1, 3), (1, 4, 3, 2), (3, 1, 2, 4), (4, 2, 3, 1)]


@pytest.mark.parametrize("dtk", KINDS)
def test_two_dimensional_paths_bit_exact(xt, dev, dtk):
    for i, dims in enumerate(TWO_D_SHAPES):
        x = rand_host(dtk, int(np.prod(dims)), 40 + i)
        for perm in TWO_D_PERMS:
            ref = O.permute(x, dims, perm)
            got = gpu_permute(xt, dev, x, dims, perm)
            assert np.array_equal(got.view(np.uint8), ref.view(np.uint8)), (dims, perm)
            if dtk in (O.C4, O.C8):  # conjugating stores (element-wise functor) on the same paths
                got = gpu_permute(xt, dev, x, dims, perm, conj_bits=1)
                assert np.array_equal(got.view(np.uint8), O.permute(x, dims, perm, conj=True).view(np.uint8))


@pytest.mark.parametrize("dtk", [O.R4, O.R8])
def test_two_dimensional_paths_permute_add(xt, dev, dtk):
    # the fused permute+add functor (element-wise stores) on the same paths
    for i, dims in enumerate(TWO_D_SHAPES[:3]):
        vol = int(np.prod(dims))
        l = rand_host(dtk, vol, 60 + i)
        for perm in TWO_D_PERMS:
            d0 = rand_host(dtk, vol, 70 + i)
            ref = O.tensor_add(list(perm), d0.copy(), l, dims, 0.37)
            dd, ld = dev.put(d0), dev.put(l)
            xt.tensor_add(dtk, dims, perm, dd.data_ptr(), ld.data_ptr(), 0.37, 0, dev.stream())
            got = dev.get(dd, d0.dtype, vol)
            assert np.array_equal(got.view(np.uint8), ref.view(np.uint8)), (dims, perm)


@pytest.mark.parametrize("dtk,dims,perm", [(O.R8, [64, 64, 48, 32], (2, 3, 1, 4)),
                                           (O.R4, [96, 80, 60, 40], (3, 4, 1, 2)),
                                           (O.C4, [64, 64, 48, 32], (4, 3, 2, 1)),
                                           (O.R4, [96, 96, 40, 30], (1, 2, 4, 3))])  # long rows: bulk kernel tried
def test_measured_plan_choice_bit_exact(xt, dev, dtk, dims, perm):
    """Copies of 32 MB and more time a few plans on their first call and keep
    the fastest: the first (timing) call and the later (cached) ones all give
    the oracle's bits."""
    x = rand_host(dtk, int(np.prod(dims)), 91)
    ref = O.permute(x, dims, perm).view(np.uint8)
    for _ in range(2):
        assert np.array_equal(gpu_permute(xt, dev, x, dims, perm).view(np.uint8), ref)
    if dtk == O.C4:
        got = gpu_permute(xt, dev, x, dims, perm, conj_bits=1)
        assert np.array_equal(got.view(np.uint8), O.permute(x, dims, perm, conj=True).view(np.uint8))


def test_skewed_extents(xt, dev):
    for dims, perm in [([3, 300, 250], [3, 1, 2]), ([2, 90, 90, 9], [4, 3, 2, 1]), ([700, 7, 5, 40], [2, 4, 1, 3]),
                       ([6, 5, 4, 3, 2, 30], [6, 1, 5, 2, 4, 3])]:
        for dtk in (O.R4, O.R8):
            x = rand_host(dtk, int(np.prod(dims)), 5)
            assert np.array_equal(gpu_permute(xt, dev, x, dims, perm), O.permute(x, dims, perm)), (dims, perm)


def test_rank0_and_volume1(xt, dev):
    x = np.array([3.25], dtype=np.float64)
    assert np.array_equal(gpu_permute(xt, dev, x, [], []), x)
    assert np.array_equal(gpu_permute(xt, dev, x, [1, 1, 1], [3, 1, 2]), x)


@pytest.mark.parametrize("dtk,dims,perm", [
    (O.R8, [76, 76, 76, 76], [3, 1, 4, 2]),
    (O.R4, [90, 90, 90, 90], [4, 3, 2, 1]),
    (O.R8, [18, 18, 18, 18, 18, 18], [6, 2, 4, 1, 5, 3]),
    (O.R4, [5, 1900, 1900, 4], [2, 4, 1, 3]),
])
def test_full_size_round_trip(xt, dev, dtk, dims, perm):
    """256 MiB-class tensors: permute then inverse-permute returns the input
    bit for bit, and the permuted tensor holds the same multiset of words."""
    import torch
    vol = int(np.prod(dims))
    es = {O.R4: 4, O.R8: 8}[dtk]
    a = torch.empty(vol * es, dtype=torch.uint8, device="cuda")
    b = torch.empty_like(a)
    c = torch.empty_like(a)
    xt.fill_uniform(dtk, vol, a.data_ptr(), 1234, stream=dev.stream())
    xt.tensor_copy(dtk, dims, perm, a.data_ptr(), b.data_ptr(), 0, dev.stream())
    inv = [0] * len(perm)
    for i, p in enumerate(perm):
        inv[p - 1] = i + 1
    xt.tensor_copy(dtk, O.permuted_dims(dims, perm), inv, b.data_ptr(), c.data_ptr(), 0, dev.stream())
    torch.cuda.synchronize()
    assert torch.equal(a, c)
    wd = torch.int32 if es == 4 else torch.int64
    assert torch.equal(torch.sort(a.view(wd)).values, torch.sort(b.view(wd)).values)
