"""GPU: two host threads contracting at the same time on two streams of one
GPU.  Every call builds its own tensor-core parameter block and scratch, and
the per-call statistics are kept per thread, so neither thread's results nor
its statistics may see the other's (each is checked against the
double-double oracle, and against its own single-threaded run bit for bit)."""
import threading

import numpy as np
import pytest

import exatensor_b200 as XB
import oracle as O
from tests.test_gpu_contract import oracle_dd

pytestmark = pytest.mark.gpu


def test_two_threads_two_streams(xt):
    import torch
    cases = [("D(i,j)+=L(k,i)*R(k,j)", [640, 512], [1024, 640], [1024, 512], 1),
             ("D(a,b,c)+=L(k,a,b)*R(c,k)", [24, 20, 300], [700, 24, 20], [300, 700], 2)]
    data = []
    for pat, dd, ld, rd, seed in cases:
        vol = lambda d: int(np.prod(d))
        l = O.splitmix64_uniform(vol(ld), seed)
        r = O.splitmix64_uniform(vol(rd), seed + 10)
        ref = oracle_dd(pat, np.zeros(vol(dd)), dd, l, ld, r, rd, 1.0, False)
        data.append((pat, dd, ld, rd, l, r, ref))

    def run(i, out, reps):
        pat, dd, ld, rd, l, r, ref = data[i]
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            lt = torch.from_numpy(l).cuda(non_blocking=False)
            rt = torch.from_numpy(r).cuda()
            res = []
            for _ in range(reps):
                dt = torch.zeros(int(np.prod(dd)), dtype=torch.float64, device="cuda")
                xt.tensor_contract(pat, O.R8, dd, dt.data_ptr(), ld, lt.data_ptr(), rd, rt.data_ptr(), 1.0,
                                   accumulative=False, plan=xt.make_plan(XB.METHOD_FUSED), stream=s.cuda_stream)
                st = xt.last_contract_stats()
                s.synchronize()
                res.append((dt.cpu().numpy(), st.m, st.n, st.k, st.method))
            out[i] = res

    # single-threaded reference runs
    alone = [None, None]
    for i in range(2):
        run(i, alone, 1)
    # both at once, several calls each
    both = [None, None]
    th = [threading.Thread(target=run, args=(i, both, 6)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    xt.device_check(None)
    for i in range(2):
        ref = data[i][6]
        want = alone[i][0]
        assert O.rel_frobenius(want[0], ref) <= 1e-12
        for got, m, n, k, method in both[i]:
            assert method == XB.METHOD_FUSED and (m, n, k) == want[1:4]
            assert np.array_equal(got.view(np.uint8), want[0].view(np.uint8))
