"""GPU parity: the fused permute+add (tb_tensor_add), init, scale and the seeded
fill are bit-exact against the oracle's restatements of tensor_block_add /
cpu_tensor_block_add (TALSH/tensor_algebra_cpu.F90:3312, TALSH/talshf.F90:1857),
tensor_block_init (:955) and tensor_block_scale (:1821).  The deterministic
norms agree with the oracle's sums to 1e-12 relative (FP64 summation order
differs) and repeat bit for bit."""
import itertools
import random

import numpy as np
import pytest

import oracle as O
from tests.test_gpu_permute import rand_host

pytestmark = pytest.mark.gpu
KINDS = [O.R4, O.R8, O.C4, O.C8]


@pytest.mark.parametrize("dtk", KINDS)
@pytest.mark.parametrize("scale", [1.0, 0.37, -2.5 + 0.75j])
def test_permute_add_bit_exact(xt, dev, dtk, scale):
    dims = [6, 5, 4, 7]
    vol = int(np.prod(dims))
    l = rand_host(dtk, vol, 1)
    for perm in list(itertools.permutations([1, 2, 3, 4]))[::5] + [(1, 2, 3, 4)]:
        d0 = rand_host(dtk, vol, 2)
        for conj_bits in ([0, 2, 3] if dtk in (O.C4, O.C8) else [0]):
            ref = O.tensor_add(list(perm), d0.copy(), l, dims, scale, conj_bits)
            dd = dev.put(d0)
            ld = dev.put(l)
            xt.tensor_add(dtk, dims, perm, dd.data_ptr(), ld.data_ptr(), scale, conj_bits, dev.stream())
            got = dev.get(dd, d0.dtype, vol)
            assert np.array_equal(got.view(np.uint8), ref.view(np.uint8)), (perm, conj_bits)


@pytest.mark.parametrize("dtk", KINDS)
def test_add_random_shapes(xt, dev, dtk):
    rng = random.Random(9)
    for case in range(15):
        rank = rng.randint(1, 5)
        dims = [rng.choice([1, 2, 3, 8, 17, 33]) for _ in range(rank)]
        perm = list(range(1, rank + 1)); rng.shuffle(perm)
        vol = int(np.prod(dims))
        l = rand_host(dtk, vol, case); d0 = rand_host(dtk, vol, 100 + case)
        ref = O.tensor_add(perm, d0.copy(), l, dims, 0.5)
        dd = dev.put(d0); ld = dev.put(l)
        xt.tensor_add(dtk, dims, perm, dd.data_ptr(), ld.data_ptr(), 0.5, 0, dev.stream())
        assert np.array_equal(dev.get(dd, d0.dtype, vol).view(np.uint8), ref.view(np.uint8)), (dims, perm)


@pytest.mark.parametrize("dtk", KINDS)
def test_init_and_scale_bit_exact(xt, dev, dtk):
    vol = 100003
    x = rand_host(dtk, vol, 4)
    d = dev.put(x)
    xt.tensor_scale(dtk, vol, d.data_ptr(), 0.3 - 0.2j, dev.stream())
    ref = O.scale(x.copy(), 0.3 - 0.2j)
    assert np.array_equal(dev.get(d, x.dtype, vol).view(np.uint8), ref.view(np.uint8))
    xt.tensor_init(dtk, vol, d.data_ptr(), 1.5 + 2.0j, dev.stream())
    ref = O.init(x.copy(), 1.5 + 2.0j)
    assert np.array_equal(dev.get(d, x.dtype, vol).view(np.uint8), ref.view(np.uint8))


@pytest.mark.parametrize("dtk", KINDS)
def test_norms(xt, dev, dtk):
    vol = 1000001
    x = rand_host(dtk, vol, 6)
    d = dev.put(x)
    for which, ref in ((1, O.norm1(x)), (2, O.norm2sq(x))):
        a = xt.tensor_norm(dtk, vol, d.data_ptr(), which, dev.stream())
        b = xt.tensor_norm(dtk, vol, d.data_ptr(), which, dev.stream())
        assert a == b  # deterministic
        assert abs(a - ref) <= 1e-12 * ref


@pytest.mark.parametrize("dtk", KINDS)
def test_fill_uniform_matches_generator(xt, dev, dtk):
    vol = 50000
    d = dev.empty(vol * {O.R4: 4, O.R8: 8, O.C4: 8, O.C8: 16}[dtk])
    xt.fill_uniform(dtk, vol, d.data_ptr(), 77, stream=dev.stream())
    assert np.array_equal(dev.get(d, O.NP_DTYPE[dtk], vol), rand_host(dtk, vol, 77))
