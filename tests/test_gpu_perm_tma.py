"""GPU parity of the TMA-staged permutation kernel (tb_perm_tma.cuh): with
TB_PERM_TMA=1 every permutation whose layout allows it runs through
cp.async.bulk.tensor box loads, and must be bit-identical to the oracle's
restatement of tensor_block_copy (TALSH/tensor_algebra_cpu.F90:3151,
:7699-7940): every data kind, all 24 rank-4 permutations, edge boxes along
both box dimensions, ranks 2, 3 and 5, conjugation.  The switch is read once
per process, so the cases run in a child process; its trace lines show that
the TMA kernel did run."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

# (data kind, extents): every input stride of dims >= 1 is a multiple of 16 bytes
CASES = [
    (8, [40, 36, 20, 12]), (4, [36, 44, 20, 12]), (18, [12, 20, 8, 6]), (14, [16, 20, 8, 6]),
    (4, [100, 300, 6]), (8, [150, 130, 3]), (4, [300, 260]), (8, [16, 8, 12, 4, 20]),
]


def child():
    import itertools

    import numpy as np

    sys.path.insert(0, ROOT)
    import exatensor_b200 as XB
    import oracle as O
    from tests.conftest import Dev
    from tests.test_gpu_permute import gpu_permute, rand_host

    XB.device_init(0)
    bad = []
    n = 0
    for dtk, dims in CASES:
        x = rand_host(dtk, int(np.prod(dims)), 17)
        perms = list(itertools.permutations(range(1, len(dims) + 1)))
        if len(perms) > 24:
            perms = perms[::5]
        for perm in perms:
            for conj in ((0, 2) if dtk in (14, 18) else (0,)):
                got = gpu_permute(XB, Dev, x, dims, perm, conj_bits=conj)
                ref = O.permute(np.conj(x) if conj else x, dims, perm)
                n += 1
                if not np.array_equal(got.view(np.uint8), ref.view(np.uint8)):
                    bad.append([dtk, dims, list(perm), conj])
    XB.device_check(Dev.stream())
    print(json.dumps({"cases": n, "bad": bad}))


def test_tma_staged_permutations_bit_exact():
    env = dict(os.environ, TB_PERM_TMA="1", TB_PERM_TRACE="1")
    r = subprocess.run([sys.executable, "-c", "import tests.test_gpu_perm_tma as t; t.child()"], cwd=ROOT,
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["cases"] > 150 and out["bad"] == [], out["bad"][:10]
    assert r.stderr.count("kernel=tma") >= 100  # the TMA kernel ran for most cases
