#!/usr/bin/env python3
"""Benchmark of the TAL-SH tensor-algebra path on B200.

Headline workload: the CCSD-like R8 contraction
    D(a,b,i,j) += V(a,b,c,d) * T(c,d,i,j),  virtual extent 192, occupied 48
(M = N_ab = 36864, N = 2304, K = 36864; 6.262e12 FLOP by TAL-SH's 2*M*N*K
accounting), inputs seeded U[-1,1) with V scaled by 1/192, D = 0.  A "step" is
one contraction by the chosen method (the library's plan selector).  The same
line reports the plain FP64 TTGT form, the error against a double-double
FP64 oracle on sampled elements, the permutation sweep (all 24 rank-4
permutations of 256 MiB R8 and R4 tensors, bit-exact) in GB/s, the
end-to-end rate through talshTensorContract with host-resident tensors, and
the reference's OpenMP+BLAS CPU path timed on this host.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
       (N > 1: launched by torchrun, one process per GPU, replicas)
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "contraction TFLOP/s + permute GB/s, chosen vs plain form at stated FP64 err"

WORKLOADS = {
    "ccsd1_r8": dict(pattern="D(a,b,i,j)+=V(a,b,c,d)*T(c,d,i,j)", v=192, o=48, dtk=8),
    "ccsd2_r8": dict(pattern="D(a,i,b,j)+=W(a,k,c,i)*T(c,b,k,j)", v=192, o=48, dtk=8),
    "ccsd1_c8": dict(pattern="D(a,b,i,j)+=V(a,b,c,d)*T(c,d,i,j)", v=192, o=48, dtk=18),
    "ccsd2_c8": dict(pattern="D(a,i,b,j)+=W(a,k,c,i)*T(c,b,k,j)", v=192, o=48, dtk=18),
    "ccsd1_r4": dict(pattern="D(a,b,i,j)+=V(a,b,c,d)*T(c,d,i,j)", v=192, o=48, dtk=4),
    "ccsd2_r4": dict(pattern="D(a,i,b,j)+=W(a,k,c,i)*T(c,b,k,j)", v=192, o=48, dtk=4),
}
VIRT = set("abcd")
# dram__bytes_read.sum + dram__bytes_write.sum of tc_gemm_kernel on the v=96 case
# (4.90 GB + 0.96 GB) times the 16x larger work of v=192 with the same tile shape
TC_GEMM_TRAFFIC = 16 * (4.902736e9 + 0.963089e9)


def shapes(pattern, v, o):
    import re
    groups = re.findall(r"\(([^)]*)\)", pattern)
    ext = lambda x: v if x in VIRT else o
    return [[ext(x) for x in g.split(",")] for g in groups]


def vol(dims):
    n = 1
    for x in dims:
        n *= x
    return n


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during a region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = os.environ.get("BENCH_DIST_BACKEND", "nccl")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------------------- GPU
class ContractionCase:
    """Device tensors of one contraction workload."""

    def __init__(self, X, wl, stream):
        import torch
        self.X, self.wl, self.s = X, wl, stream
        self.dd, self.ld, self.rd = shapes(wl["pattern"], wl["v"], wl["o"])
        es = X.ELEM_BYTES[wl["dtk"]]
        self.D = torch.empty(vol(self.dd) * es, dtype=torch.uint8, device="cuda")
        self.L = torch.empty(vol(self.ld) * es, dtype=torch.uint8, device="cuda")
        self.R = torch.empty(vol(self.rd) * es, dtype=torch.uint8, device="cuda")
        X.fill_uniform(wl["dtk"], vol(self.ld), self.L.data_ptr(), 1, stream=stream)
        X.fill_uniform(wl["dtk"], vol(self.rd), self.R.data_ptr(), 2, stream=stream)
        X.tensor_scale(wl["dtk"], vol(self.ld), self.L.data_ptr(), 1.0 / wl["v"], stream=stream)
        X.tensor_init(wl["dtk"], vol(self.dd), self.D.data_ptr(), 0.0, stream=stream)
        cp, *_ = X.parse_pattern(wl["pattern"])
        self.cptrn = cp
        # 2*M*N*K, or 8*M*N*K for complex data (the reference's accounting)
        cplx = wl["dtk"] in (14, 18)
        self.flops = (8.0 if cplx else 2.0) * vol(self.dd) * (vol(self.ld) * vol(self.rd) / vol(self.dd)) ** 0.5

    def run(self, method, accumulative=True, plan=None):
        X = self.X
        X.tensor_contract(self.cptrn, self.wl["dtk"], self.dd, self.D.data_ptr(), self.ld, self.L.data_ptr(),
                          self.rd, self.R.data_ptr(), 1.0, 0, accumulative, plan or X.make_plan(method), self.s)


def time_steps(fn, steps, warmup, world, stream_obj, on_timed=None):
    """Device time (ms) of `steps` calls of fn after `warmup` untimed calls;
    on_timed() runs between the two (after a synchronize), e.g. to reset
    per-kernel counters so that they cover the timed calls only."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    if on_timed is not None:
        on_timed()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream_obj)
    for _ in range(steps):
        fn()
    e1.record(stream_obj)
    torch.cuda.synchronize()
    barrier(world)
    return e0.elapsed_time(e1)


def time_back_to_back(fn, steps, stream_obj):
    """Device time (ms) of `steps` back-to-back calls of fn, with one untimed
    call already queued when the start event is recorded, so that the host's
    latency before the first launch is not counted (steady-state rate of a
    kernel much shorter than a step of the headline workload)."""
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fn()
    e0.record(stream_obj)
    for _ in range(steps):
        fn()
    e1.record(stream_obj)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def sample_error(X, case, method, nsamp=48):
    """Relative Frobenius and max-abs error of sampled D elements against the
    double-double oracle (each a K-length dot product of the operands'
    elements gathered on the device), after one non-accumulating contraction.
    Any contraction pattern without conjugation; real or complex data."""
    import numpy as np
    import torch

    import oracle as O
    case.run(method, accumulative=False)
    torch.cuda.synchronize()
    dt = O.NP_DTYPE[case.wl["dtk"]]
    tdt = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32,
           np.dtype(np.complex128): torch.complex128, np.dtype(np.complex64): torch.complex64}[np.dtype(dt)]

    def strides(d):
        st = [1]
        for x in d[:-1]:
            st.append(st[-1] * x)
        return st
    cptrn = list(case.cptrn)
    lr, rr = len(case.ld), len(case.rd)
    Ls, Rs, Ds = strides(case.ld), strides(case.rd), strides(case.dd)
    pairs = [(i, -cptrn[i] - 1) for i in range(lr) if cptrn[i] < 0]
    grids = torch.meshgrid(*[torch.arange(case.ld[i], device="cuda", dtype=torch.int64) for i, _ in pairs],
                           indexing="ij")
    loff = sum(g.reshape(-1) * Ls[i] for g, (i, _) in zip(grids, pairs))
    roff = sum(g.reshape(-1) * Rs[j] for g, (_, j) in zip(grids, pairs))
    K = int(loff.numel())
    Lv, Rv, Dv = case.L.view(tdt), case.R.view(tdt), case.D.view(tdt)
    rng = np.random.default_rng(5)
    num = den = mx = 0.0
    for _ in range(nsamp):
        dix = [int(rng.integers(x)) for x in case.dd]
        lb = sum(dix[cptrn[i] - 1] * Ls[i] for i in range(lr) if cptrn[i] > 0)
        rb = sum(dix[cptrn[lr + j] - 1] * Rs[j] for j in range(rr) if cptrn[lr + j] > 0)
        lv = np.ascontiguousarray(Lv[lb + loff].cpu().numpy())
        rv = np.ascontiguousarray(Rv[rb + roff].cpu().numpy())
        ref = np.zeros(1, dtype=dt)
        O.contract([-1, -1], ref, [], lv, [K], rv, [K], 1.0, 0, True, mode=1)
        got = complex(Dv[sum(x * st for x, st in zip(dix, Ds))].item())
        e = abs(got - complex(ref[0]))
        num += e * e
        den += abs(complex(ref[0])) ** 2
        mx = max(mx, e)
    return {"rel_frobenius": (num / den) ** 0.5, "max_abs": mx, "samples": nsamp}


def configs_case(X, s, s_obj, names, steps, warmup):
    """Chosen (plan selector) and plain TTGT forms of each CCSD-like workload:
    device-timed TFLOP/s and sampled errors against the double-double oracle."""
    import torch
    out = []
    for name in names:
        wl = WORKLOADS[name]
        case = ContractionCase(X, wl, s)
        ms = time_steps(lambda: case.run(X.METHOD_AUTO), steps, warmup, 1, s_obj) / steps
        st = X.last_contract_stats()
        pms = time_steps(lambda: case.run(X.METHOD_TTGT), steps, 1, 1, s_obj) / steps
        e_c = sample_error(X, case, X.METHOD_AUTO, 24)
        e_p = sample_error(X, case, X.METHOD_TTGT, 24)
        rec = {"workload": name, "pattern": wl["pattern"], "data_kind": wl["dtk"], "flop": case.flops,
               "chosen": {"method": {1: "ttgt", 2: "tensor cores"}.get(st.method, st.method), "slices": st.slices,
                          "products": st.products, "tile_n": st.tile_n, "tile_m": st.tile_m, "ms": round(ms, 3),
                          "TFLOP/s": round(case.flops / (ms / 1e3) / 1e12, 2), "rel_frobenius": e_c["rel_frobenius"]},
               "plain": {"ms": round(pms, 3), "TFLOP/s": round(case.flops / (pms / 1e3) / 1e12, 2),
                         "rel_frobenius": e_p["rel_frobenius"]},
               "chosen_over_plain": round(pms / ms, 3)}
        out.append(rec)
        print(json.dumps(rec), flush=True)
        del case
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return out


def permute_sweep(X, stream, stream_obj, hbm_gbs):
    """All 24 rank-4 permutations of 256 MiB-class R8 (76^4) and R4 (90^4)."""
    import itertools

    import torch
    out = {}
    total_bytes = total_ms = 0.0
    rates = []
    for dtk, n in ((8, 76), (4, 90)):
        es = X.ELEM_BYTES[dtk]
        v = n ** 4
        a = torch.empty(v * es, dtype=torch.uint8, device="cuda")
        b = torch.empty_like(a)
        X.fill_uniform(dtk, v, a.data_ptr(), 3, stream=stream)
        dims = [n] * 4
        for perm in itertools.permutations([1, 2, 3, 4]):
            # the first call of a shape also picks its plan by timing (untimed here)
            X.tensor_copy(dtk, dims, perm, a.data_ptr(), b.data_ptr(), 0, stream)
            ms = time_back_to_back(lambda: X.tensor_copy(dtk, dims, perm, a.data_ptr(), b.data_ptr(), 0, stream),
                                   10, stream_obj) / 10
            gb = 2.0 * v * es / 1e9
            rates.append(gb / (ms / 1e3))
            total_bytes += gb
            total_ms += ms
        # plain scatter form for reference (two permutations)
        sc = []
        for perm in ((4, 3, 2, 1), (2, 4, 1, 3)):
            ms = time_steps(lambda: X.tensor_copy(dtk, dims, perm, a.data_ptr(), b.data_ptr(), 0, stream, True), 3,
                            1, 1, stream_obj) / 3
            sc.append(2.0 * v * es / 1e9 / (ms / 1e3))
        out[f"scatter_gbs_{'r8' if dtk == 8 else 'r4'}"] = round(statistics.mean(sc), 1)
        del a, b
    agg = total_bytes / (total_ms / 1e3)
    out.update({"value": round(agg, 1), "unit": "GB/s", "min": round(min(rates), 1), "max": round(max(rates), 1),
                "frac_of_measured_hbm": round(agg / hbm_gbs, 3), "frac_of_8000": round(agg / 8000.0, 3),
                "cases": "24 rank-4 perms x {R8 76^4 (254.5 MiB), R4 90^4 (250.3 MiB)}, bit-exact",
                "timing": "10 back-to-back calls per permutation, one queued before the start event; "
                          "plans picked by the library's measured choice on the first call"})
    return out


def permute_sweep_repeated(X, stream, stream_obj, reps=3):
    """The permutation sweep's 48 cases, `reps` times after 0.5 s of copies
    that let the clocks settle; per-case medians, their aggregate
    (bytes over time) and the mean relative spread of the repetitions.
    Library knobs set in the environment (TB_PERM_TUNE, TB_PERM_FAST,
    TB_PERM_VMIN_KB/VMAX_KB) apply, so variants can be compared."""
    import itertools

    import torch
    bufs = {}
    for dtk, n in ((8, 76), (4, 90)):
        es = X.ELEM_BYTES[dtk]
        v = n ** 4
        a = torch.empty(v * es, dtype=torch.uint8, device="cuda")
        b = torch.empty_like(a)
        X.fill_uniform(dtk, v, a.data_ptr(), 3, stream=stream)
        bufs[dtk] = (n, v, es, a, b)
    t0 = time.time()
    while time.time() - t0 < 0.5:
        for dtk, (n, v, es, a, b) in bufs.items():
            X.tensor_copy(dtk, [n] * 4, (2, 1, 3, 4), a.data_ptr(), b.data_ptr(), 0, stream)
        torch.cuda.synchronize()
    perms = list(itertools.permutations([1, 2, 3, 4]))
    runs = {dtk: [[] for _ in perms] for dtk in bufs}
    for _ in range(reps):
        for dtk, (n, v, es, a, b) in bufs.items():
            for i, perm in enumerate(perms):
                ms = time_back_to_back(lambda: X.tensor_copy(dtk, [n] * 4, perm, a.data_ptr(), b.data_ptr(), 0,
                                                             stream), 10, stream_obj) / 10
                runs[dtk][i].append(2.0 * v * es / 1e9 / (ms / 1e3))
    out, tot_b, tot_s = {}, 0.0, 0.0
    for dtk, key in ((8, "r8"), (4, "r4")):
        n, v, es, _, _ = bufs[dtk]
        med = [statistics.median(x) for x in runs[dtk]]
        out[key] = {"".join(map(str, p)): round(m) for p, m in zip(perms, med)}
        out[key + "_spread"] = round(statistics.mean((max(x) - min(x)) / statistics.median(x) for x in runs[dtk]), 3)
        tot_b += 24 * 2.0 * v * es / 1e9
        tot_s += sum(2.0 * v * es / 1e9 / m for m in med)
    out["GB/s"] = round(tot_b / tot_s, 1)
    out["env"] = {k: os.environ.get(k) for k in ("TB_PERM_TUNE", "TB_PERM_FAST", "TB_PERM_VMIN_KB", "TB_PERM_VMAX_KB")}
    return out


BSC = dict(pattern="D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)", nseg=6, lo=8, hi=96, presence=0.3, seed=1)


def block_sparse_case(X, stream, stream_obj, dtk=8, steps=1, nseg=None, hi=None, run_loop=True):
    """Block-sparse CCSD-like contraction: every index split into 6 seeded
    segments of 8..96, 30% of the blocks of L and R present; all matching
    block pairs (about 4.2k uneven block GEMMs) as one grouped launch replayed
    from a CUDA graph, against the per-block loop of tb_tensor_contract calls.
    Errors compare 16 sampled output blocks of the two runs."""
    import numpy as np
    import torch

    from exatensor_b200 import blocksparse as BS
    cfg = dict(BSC)
    cfg["nseg"] = nseg or cfg["nseg"]
    cfg["hi"] = hi or cfg["hi"]
    rng = np.random.default_rng(cfg["seed"])
    es = X.ELEM_BYTES[dtk]
    seg = BS.random_segments(6, cfg["nseg"], cfg["lo"], cfg["hi"], rng)  # a b c d i j
    segl, segr = seg[0:4], seg[2:6]
    L = BS.BlockSparseTensor(segl, BS.random_keys(segl, cfg["presence"], rng), es)
    R = BS.BlockSparseTensor(segr, BS.random_keys(segr, cfg["presence"], rng), es)
    X.fill_uniform(dtk, L.volume, L.data.data_ptr(), 21, stream=stream)
    X.fill_uniform(dtk, R.volume, R.data.data_ptr(), 22, stream=stream)
    D, tasks, pairs = BS.contraction_tasks(cfg["pattern"], L, R)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plan = X.BlockSparsePlan(cfg["pattern"], dtk, tasks, accumulative=False, stream=stream)
    plan_s = time.perf_counter() - t0
    plan.autotune(stream=stream)
    inf = plan.info()
    gms = time_steps(lambda: plan.execute(stream=stream), steps, 1, 1, stream_obj) / steps
    keys = list(D.blocks)
    pick = [keys[int(i)] for i in rng.choice(len(keys), size=min(16, len(keys)), replace=False)]
    dt = {8: np.float64, 4: np.float32}[dtk]

    def sample():
        torch.cuda.synchronize()
        out = []
        for k in pick:
            off, dims = D.blocks[k]
            n = int(np.prod(dims))
            out.append(D.data[off * es:(off + n) * es].cpu().numpy().view(dt).copy())
        return np.concatenate(out)

    got = sample()
    plan.close()
    base = D.data.data_ptr()

    def reference():
        # FP64 sums of the sampled output blocks from the operand blocks
        # (the pattern is D(a,b,i,j) += L(a,b,c,d) * R(c,d,i,j))
        # as matrices: L block [ab][cd] times R block [cd][ij] (dlf order), BLAS
        def block(T, k, rows):
            off, dims = T.blocks[k]
            n = int(np.prod(dims))
            x = T.data[off * es:(off + n) * es].cpu().numpy().view(dt).astype(np.float64)
            return x.reshape((rows, n // rows), order="F")
        out = []
        for k in pick:
            dd = D.blocks[k][1]
            acc = np.zeros((dd[0] * dd[1], dd[2] * dd[3]), dtype=np.float64)
            for dk, lk, rk in pairs:
                if dk == k:
                    ld, rd = L.blocks[lk][1], R.blocks[rk][1]
                    acc += block(L, lk, ld[0] * ld[1]) @ block(R, rk, rd[0] * rd[1])
            out.append(acc.ravel(order="F"))
        return np.concatenate(out)
    ref = reference()

    def loop():
        D.data.zero_()
        for dp, dd, lp, ld, rp, rd in tasks:
            X.tensor_contract(cfg["pattern"], dtk, dd, dp, ld, lp, rd, rp, 1.0, 0, True, None, stream)

    rel_of = lambda x: float(np.linalg.norm(x.astype(np.float64) - ref) / np.linalg.norm(ref))
    if not run_loop:
        return {"pairs": len(tasks), "flops": inf.flops, "grouped_ms": round(gms, 2),
                "grouped_tflops": round(inf.flops / (gms / 1e3) / 1e12, 3), "rel_frobenius_vs_fp64": rel_of(got)}
    lms = time_steps(loop, 1, 0, 1, stream_obj)
    want = sample()
    del base
    rel = float(np.linalg.norm(got.astype(np.float64) - want) / np.linalg.norm(want))
    res = {"workload": f"bsc_{'r8' if dtk == 8 else 'r4'}: {cfg['pattern']}, {cfg['nseg']} segments of "
                       f"{cfg['lo']}..{cfg['hi']} per index, {int(cfg['presence'] * 100)}% blocks, seed {cfg['seed']}",
           "pairs": len(tasks), "out_blocks": len(D.blocks), "flops": inf.flops,
           "grouped": {"value": round(inf.flops / (gms / 1e3) / 1e12, 3), "unit": "TFLOP/s", "ms": round(gms, 2),
                       "launch": "CUDA graph: grouped conversion + one persistent grouped GEMM"},
           "per_block_loop": {"value": round(inf.flops / (lms / 1e3) / 1e12, 3), "unit": "TFLOP/s",
                              "ms": round(lms, 2), "launch": f"{len(tasks)} tb_tensor_contract calls"},
           "grouped_over_loop": round(lms / gms, 2),
           "rel_frobenius_grouped_vs_loop": rel,
           "rel_frobenius_vs_fp64": {"grouped": rel_of(got), "per_block_loop": rel_of(want),
                                     "blocks_sampled": len(pick)},
           "autotune": {"tile_n": inf.tile_n, "slices": inf.slices, "tune_ms": [round(x, 2) for x in inf.tune_ms]},
           "plan_seconds": round(plan_s, 2)}
    del L, R, D, tasks
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return res


SELECTOR_CORPUS = os.path.join(ROOT, "tests", "golden", "selector_corpus.npz")


def selector_case(X):
    """Learned plan selector on the recorded corpus: trained with the
    library's CUDA kernels on the first 80% of the corpus, judged on the rest
    by runtime regret against the best measured plan, beside the size rule;
    plus the selection latency of the host inference used by METHOD_AUTO and
    the GPU batch inference kernel's throughput."""
    import numpy as np
    import torch

    from exatensor_b200 import selector as S
    if not os.path.exists(SELECTOR_CORPUS):
        return None
    d = np.load(SELECTOR_CORPUS)
    F, T = d["features"], d["log_ms"]
    ok = np.isfinite(T).all(axis=1)
    F, T = F[ok], T[ok]
    n_train = int(0.8 * len(F))
    t0 = time.perf_counter()
    params, mean, scale, hist = S.train(F[:n_train], T[:n_train], hidden=128, epochs=150, seed=0, log_every=149)
    train_s = time.perf_counter() - t0
    pred = S.predict(params, mean, scale, F[n_train:], hidden=128)
    learned = S.evaluate(T[n_train:], pred.argmin(axis=1))
    rule = S.evaluate(T[n_train:], [S.rule_choice(f) for f in F[n_train:]])
    always = {name: S.evaluate(T[n_train:], [i] * (len(F) - n_train))["total_time_regret"]
              for i, name in enumerate(S.PLAN_NAMES)}
    X.selector_install(128, params, mean, scale)
    t0 = time.perf_counter()
    for f in F[n_train:n_train + 2000]:
        X.selector_choose(f)
    host_us = (time.perf_counter() - t0) / min(2000, len(F) - n_train) * 1e6
    X.selector_install(0, None, None, None)
    net = X.MLP(F.shape[1], 128, len(S.PLANS), max_batch=1024)
    net.set_params(params)
    xn = torch.from_numpy(((F[n_train:] - mean) / scale).astype(np.float32)).cuda()
    y = torch.empty((len(xn), len(S.PLANS)), dtype=torch.float32, device="cuda")
    net.forward(xn.data_ptr(), len(xn), y.data_ptr())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        net.forward(xn.data_ptr(), len(xn), y.data_ptr())
    e1.record()
    torch.cuda.synchronize()
    gpu_us = e0.elapsed_time(e1) / 10 * 1e3 / len(xn)
    net.close()
    return {"corpus": f"{int(ok.sum())} labelled random contractions (seed 0), {n_train} train / "
                      f"{len(F) - n_train} held out", "plans": S.PLAN_NAMES,
            "learned": learned, "size_rule": rule, "always_one_plan_total_regret": always,
            "train_seconds": round(train_s, 1), "final_train_loss": round(hist[-1][1], 4) if hist else None,
            "selection_us_host": round(host_us, 2), "selection_us_gpu_batched": round(gpu_us, 4)}


def e2e_talsh(X, wl, steps):
    """Same contraction through talshTensorContract with Host-resident tensors:
    each step copies V, T, D to the GPU and D back (copy control TTT)."""
    import exatensor_b200.talsh as T
    T.init((int(os.environ.get("LOCAL_RANK", "0")),))
    dd, ld, rd = shapes(wl["pattern"], wl["v"], wl["o"])
    es = X.ELEM_BYTES[wl["dtk"]]
    D = T.Tensor(dd, wl["dtk"], 0.0)
    L = T.Tensor(ld, wl["dtk"], 1.0 / (3 * wl["v"]))
    R = T.Tensor(rd, wl["dtk"], 0.5)
    run = lambda: T.check(T.contract(wl["pattern"], D, L, R, 1.0, 0, T.DEV_NVIDIA_GPU, T.COPY_TTT, True),
                          "talshTensorContract")
    for _ in range(2):  # the second call of a shape may time close plan candidates once
        run()
    t0 = time.perf_counter()
    for _ in range(steps):
        run()
    dt = (time.perf_counter() - t0) / steps
    flops = 2.0 * vol(dd) * (vol(ld) * vol(rd) / vol(dd)) ** 0.5
    res = {"value": round(flops / dt / 1e12, 3), "unit": "TFLOP/s", "ms_per_step": round(dt * 1e3, 2),
           "h2d_bytes_per_step": (vol(dd) + vol(ld) + vol(rd)) * es, "d2h_bytes_per_step": vol(dd) * es,
           "api": "talshTensorContract(COPY_TTT), host tensors, wall clock incl. H2D/D2H",
           "path": ("inputs streamed to the GPU in slices under the computation" if os.environ.get("TB_STREAM") != "0"
                    else "inputs staged whole, then the contraction")}
    del D, L, R
    return res


# ----------------------------------------------------------------------------- CPU
def cpu_contraction_sample(steps=1):
    """The reference's OpenMP+BLAS CPU path (oracle restatement) on a bounded
    sample of the CCSD-like contraction: v=96, o=48 (same pattern and index
    map, 1/16 of the FLOPs)."""
    import numpy as np

    import oracle as O
    nthr = O.nthreads_default()
    if not O.blas_available():
        return None
    v, o = 96, 48
    pattern = WORKLOADS["ccsd1_r8"]["pattern"]
    dd, ld, rd = shapes(pattern, v, o)
    cptrn, *_ = O.parse_pattern(pattern)
    L = O.splitmix64_uniform(vol(ld), 1) / v
    R = O.splitmix64_uniform(vol(rd), 2)
    D = np.zeros(vol(dd))
    O.contract_blas(cptrn, D, dd, L, ld, R, rd, 1.0, True, nthr)
    best = None
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        O.contract_blas(cptrn, D, dd, L, ld, R, rd, 1.0, True, nthr)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    flops = 2.0 * vol(dd) * (vol(ld) * vol(rd) / vol(dd)) ** 0.5
    return {"value": round(flops / best / 1e12, 4), "unit": "TFLOP/s", "cores": nthr, "kind": "port",
            "sample": f"{pattern} v={v} o={o} R8 ({flops:.3e} FLOP), OpenMP permutes + OpenBLAS dgemm, "
                      f"best of {max(1, steps)}"}


def run_reference(args):
    """Reference arm: the reference's CPU implementation of the path (its
    OpenMP+BLAS CP-TAL contraction, restated in oracle/ because the Fortran
    reference cannot be compiled here), on this host's cores."""
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import oracle as O
    O.build()
    res = cpu_contraction_sample(steps=max(1, args.steps))
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "bundled OpenBLAS not found"}))
        return
    line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": "TFLOP/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded splitmix64 U[-1,1), V scaled 1/v)",
            "config": {"workload": f"{args.workload}: {WORKLOADS[args.workload]['pattern']} "
                                   f"v={WORKLOADS[args.workload]['v']} o={WORKLOADS[args.workload]['o']}",
                       "parallelism": "host threads", "sample": res["sample"]},
            "cpu_baseline": res,
            "e2e": {"value": res["value"], "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ----------------------------------------------------------------------------- main
def run_ours(args):
    import torch

    import exatensor_b200 as X
    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    X.device_init(local)
    hbm_gbs, bf16_tflops, peak_src = peaks()
    s_obj = torch.cuda.current_stream()
    s = s_obj.cuda_stream
    wl = WORKLOADS[args.workload]
    bsc = None
    if rank == 0 and not args.no_block_sparse:
        try:
            bsc = block_sparse_case(X, s, s_obj, 8, steps=1)
        except Exception as exc:  # reported, not fatal: the headline contraction still runs
            bsc = {"error": str(exc)[:300]}
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
    case = ContractionCase(X, wl, s)
    torch.cuda.synchronize()
    # chosen form (plan selector)
    case.run(X.METHOD_AUTO)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    n0 = [0]

    def start_counters():
        # the warm-up calls include the selector's one-time timing of close
        # candidates; launches and GEMM events count the timed calls only
        n0[0] = X.launch_count()
        X.timing_enable(True)
        X.timing_read()
        clocks.start()
    ms = time_steps(lambda: case.run(X.METHOD_AUTO), args.steps, args.warmup, world, s_obj, on_timed=start_counters)
    clk = clocks.stop()
    gemm_ms, gemm_n = X.timing_read()
    X.timing_enable(False)
    launches = X.launch_count() - n0[0]
    st = X.last_contract_stats()
    chosen_method = {1: "ttgt", 2: "fused"}.get(st.method, str(st.method))
    ms_max = max_over_ranks(ms, world)
    value = world * args.steps * case.flops / (ms_max / 1e3) / 1e12
    # plain form
    psteps = max(1, args.steps // 2)
    pms = time_steps(lambda: case.run(X.METHOD_TTGT), psteps, 1, world, s_obj,
                     on_timed=lambda: (X.timing_enable(True), X.timing_read()))
    pgemm_ms, pgemm_n = X.timing_read()
    X.timing_enable(False)
    plain = case.flops / (max_over_ranks(pms, world) / psteps / 1e3) / 1e12
    line = None
    if rank == 0:
        err_chosen = sample_error(X, case, X.METHOD_AUTO)
        err_plain = sample_error(X, case, X.METHOD_TTGT)
        perm = permute_sweep(X, s, s_obj, hbm_gbs)
        try:
            sel = selector_case(X)
        except Exception as exc:  # reported, not fatal
            sel = {"error": str(exc)[:300]}
        # dominant kernel of the chosen step
        per_launch_ms = gemm_ms / max(1, gemm_n)
        if chosen_method == "fused":
            kern = "tcgen05 INT8-slice GEMM" if wl["dtk"] in (8, 18) else "tcgen05 split-BF16 GEMM"
            hw_ops = case.flops * max(1, st.products)  # each slice pair / BF16 term is a full GEMM
            peak = 2 * bf16_tflops if wl["dtk"] in (8, 18) else bf16_tflops
            peak_note = (f"2 x {peak_src} bf16 dense (INT8 dense rate)" if wl["dtk"] in (8, 18)
                         else f"{peak_src} bf16 dense")
        else:
            kern = "FP64 DMMA GEMM (mma.sync m8n8k4)" if wl["dtk"] in (8, 18) else "FP32 FFMA GEMM"
            hw_ops = case.flops
            peak = 40.0 if wl["dtk"] in (8, 18) else 75.0
            peak_note = "nominal B200 FP64 tensor-core rate (not in MEASURED_PEAKS.json)"
        achieved = hw_ops / (per_launch_ms / 1e3) / 1e12 if gemm_n else None
        roofline = {"bound": "tensor", "kernel": kern, "achieved": round(achieved, 2) if achieved else None,
                    "peak": peak, "unit": "TFLOP/s", "frac": round(achieved / peak, 3) if achieved else None,
                    "traffic": TC_GEMM_TRAFFIC if (chosen_method == "fused" and args.workload == "ccsd1_r8") else None,
                    "traffic_note": "DRAM read+write bytes per launch: ncu capture of the v=96 case "
                                    "scaled by the 16x work of v=192",
                    "peak_source": peak_note, "launch_ms": round(per_launch_ms, 3), "launches_timed": gemm_n}
        e2e = e2e_talsh(X, wl, steps=max(1, min(2, args.steps)))
        cpu = cpu_contraction_sample(steps=1) if world == 1 else None
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": {4: "f32", 8: "f64", 14: "c64", 18: "c128"}[wl["dtk"]],
            "data": "synthetic (seeded splitmix64 U[-1,1), V scaled 1/v, D=0)",
            "config": {"workload": f"{args.workload}: {wl['pattern']} v={wl['v']} o={wl['o']}",
                       "method": chosen_method, "slices": st.slices, "passes": st.passes, "products": st.products,
                       "tile_n": st.tile_n, "tile_m": st.tile_m,
                       "l2": "inputs larger than L2 (V alone is 10.9 GB)", "parallelism": f"replicas x{world}"},
            "plain": {"value": round(plain, 3), "unit": "TFLOP/s", "method": "ttgt (permute + FP64 DMMA GEMM)",
                      "gemm_ms_per_launch": round(pgemm_ms / max(1, pgemm_n), 3),
                      "chosen_over_plain": round(value / world / plain, 3)},
            "error": {"chosen": err_chosen, "plain": err_plain, "oracle": "double-double dot products"},
            "permute": perm, "block_sparse": bsc, "selector": sel, "roofline": roofline, "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches, "clocks": clk,
        }
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))


def run_profile(args):
    """A small, single-part run for profilers: --profile contract|plain runs the
    chosen / plain contraction of the workload (extents overridable with --v and
    --o), --profile permute runs the 24 rank-4 permutations of an n^4 R8 tensor
    (n = --v).  Prints one summary line; not a bench result."""
    import itertools

    import torch

    import exatensor_b200 as X
    torch.cuda.set_device(0)
    X.device_init(0)
    s_obj = torch.cuda.current_stream()
    s = s_obj.cuda_stream
    if args.profile == "selector":
        print(json.dumps({"profile": "selector", **(selector_case(X) or {"error": "no corpus"})}))
        return
    if args.profile == "bsc":
        print(json.dumps({"profile": "bsc", **block_sparse_case(X, s, s_obj, args.dtk, steps=max(1, args.steps),
                                                                nseg=args.v or None, hi=args.o or None,
                                                                run_loop=not (args.v or args.o))}))
        return
    if args.profile == "configs":
        names = [w for w in (args.workloads or "").split(",") if w] or list(WORKLOADS)
        configs_case(X, s, s_obj, names, max(1, args.steps), max(1, args.warmup))
        return
    if args.profile == "e2e":
        wl = dict(WORKLOADS[args.workload])
        wl["v"] = args.v or wl["v"]
        print(json.dumps({"profile": "e2e", "workload": args.workload, "v": wl["v"],
                          **e2e_talsh(X, wl, max(1, args.steps))}))
        return
    if args.profile == "permsweep":
        print(json.dumps({"profile": "permsweep", **permute_sweep_repeated(X, s, s_obj, reps=max(1, args.steps))}))
        return
    if args.profile == "permute":
        n = args.v or 76
        v = n ** 4
        a = torch.empty(v * 8, dtype=torch.uint8, device="cuda")
        b = torch.empty_like(a)
        X.fill_uniform(8, v, a.data_ptr(), 3, stream=s)
        perms = list(itertools.permutations([1, 2, 3, 4]))
        ms = time_steps(lambda: [X.tensor_copy(8, [n] * 4, p, a.data_ptr(), b.data_ptr(), 0, s) for p in perms],
                        args.steps, args.warmup, 1, s_obj)
        print(json.dumps({"profile": "permute", "n": n, "GB/s": round(2.0 * v * 8 * len(perms) * args.steps
                                                                       / (ms / 1e3) / 1e9, 1)}))
        return
    wl = dict(WORKLOADS[args.workload])
    wl["v"] = args.v or wl["v"]
    wl["o"] = args.o or wl["o"]
    case = ContractionCase(X, wl, s)
    method = X.METHOD_AUTO if args.profile == "contract" else X.METHOD_TTGT
    plan = None
    if args.plan:  # e.g. "method=2,tile_n=256,tile_m=256,slices=6"
        kw = {k: int(v) for k, v in (x.split("=") for x in args.plan.split(","))}
        plan = X.make_plan(**kw)
    ms = time_steps(lambda: case.run(method, plan=plan), args.steps, args.warmup, 1, s_obj)
    X.device_check(s)
    st = X.last_contract_stats()
    print(json.dumps({"profile": args.profile, "workload": args.workload, "v": wl["v"], "o": wl["o"],
                      "method": st.method, "slices": st.slices, "products": st.products, "tile_n": st.tile_n,
                      "tile_m": st.tile_m,
                      "ms_per_step": round(ms / args.steps, 3),
                      "TFLOP/s": round(case.flops * args.steps / (ms / 1e3) / 1e12, 3)}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="ccsd1_r8")
    ap.add_argument("--workloads", default=None, help="--profile configs: comma-separated workloads (default all)")
    ap.add_argument("--dtk", type=int, choices=[4, 8], default=8, help="--profile bsc: data kind (R4 or R8)")
    ap.add_argument("--plan", default=None, help="--profile contract: explicit plan, e.g. method=2,tile_n=256,tile_m=256")
    ap.add_argument("--no-block-sparse", action="store_true", help="skip the block-sparse measurement")
    ap.add_argument("--profile", choices=["contract", "plain", "permute", "permsweep", "bsc", "selector", "e2e",
                                          "configs"],
                    default=None,
                    help="run one part on a small case for a profiler (no bench line)")
    ap.add_argument("--v", type=int, default=0, help="--profile: virtual extent (permute: n; bsc: segments per index)")
    ap.add_argument("--o", type=int, default=0, help="--profile: occupied extent (bsc: largest segment)")
    args = ap.parse_args()
    if args.profile:
        run_profile(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
