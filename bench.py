#!/usr/bin/env python3
"""Benchmark of the TAL-SH tensor-algebra path on B200.

Headline workload: the CCSD-like R8 contraction
    D(a,b,i,j) += V(a,b,c,d) * T(c,d,i,j),  virtual extent 192, occupied 48
(M = N_ab = 36864, N = 2304, K = 36864; 6.262e12 FLOP by TAL-SH's 2*M*N*K
accounting), inputs seeded U[-1,1) with V scaled by 1/192, D = 0.  A "step" is
one contraction by the chosen method (the library's plan selector).  The same
line reports the plain FP64 TTGT form (chosen_over_plain), the error of the
chosen D against the plain D over the whole tensor and against a
double-double FP64 oracle on 4096 sampled elements, the other five CCSD-like
configurations (R8/C8/R4, both patterns), the single-block 40^4
configuration, the permutation and add sweeps (256 MiB R8/R4 tensors of rank
2-6, uniform and skewed extents, every case checked bit for bit) in GB/s, the
block-sparse grouped launch, the learned plan selector, the tensor-core peaks
measured by the library's own probes (the roofline denominators), the
end-to-end rate through talshTensorContract with host-resident tensors, and
the reference's OpenMP+BLAS CPU path timed on this host.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
       (N > 1: launched by torchrun, one process per GPU, replicas; the line
       then holds the headline contraction only)
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
# dram__bytes_read.sum + dram__bytes_write.sum of tc_gemm_kernel (14 modular
# residues, moduli outermost, dynamic work units, B planes kept in L2) on the
# v=96 case (1.68 GB + 0.27 GB) times the 16x larger work of v=192 with the
# same tile shape
TC_GEMM_TRAFFIC = 16 * (1.683749e9 + 0.273529e9)


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


def sample_error(X, case, nsamp, seed=5, chunk=256):
    """Sampled check of the D now held by `case` (a non-accumulating
    contraction of the case's operands): `nsamp` seeded D elements, each
    against a K-long dot product with double-double accumulation (the FP64
    error oracle, oracle.dd_dot_batch).  The operand elements of each sampled
    dot product are gathered on the device.  R8 and C8 data."""
    import numpy as np
    import torch

    import oracle as O
    torch.cuda.synchronize()
    cplx = case.wl["dtk"] in (14, 18)
    tdt = torch.complex128 if cplx else torch.float64

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
    Lv, Rv, Dv = case.L.view(tdt), case.R.view(tdt), case.D.view(tdt)
    rng = np.random.default_rng(seed)
    dix = np.stack([rng.integers(0, x, nsamp) for x in case.dd], axis=1)
    zero = np.zeros(nsamp, dtype=np.int64)
    lb = zero + sum(dix[:, cptrn[i] - 1] * Ls[i] for i in range(lr) if cptrn[i] > 0)
    rb = zero + sum(dix[:, cptrn[lr + j] - 1] * Rs[j] for j in range(rr) if cptrn[lr + j] > 0)
    doff = torch.from_numpy((dix * np.array(Ds, dtype=np.int64)).sum(axis=1)).cuda()
    got = Dv[doff].cpu().numpy()
    ref = np.empty(nsamp, dtype=np.complex128 if cplx else np.float64)
    lb_t, rb_t = torch.from_numpy(lb).cuda(), torch.from_numpy(rb).cuda()
    for c0 in range(0, nsamp, chunk):
        c1 = min(nsamp, c0 + chunk)
        lv = Lv[lb_t[c0:c1, None] + loff[None, :]].cpu().numpy()
        rv = Rv[rb_t[c0:c1, None] + roff[None, :]].cpu().numpy()
        ref[c0:c1] = O.dd_dot_batch(lv, rv)
    e = np.abs(got - ref)
    return {"rel_frobenius": float(np.sqrt((e ** 2).sum() / (np.abs(ref) ** 2).sum())), "max_abs": float(e.max()),
            "samples": nsamp}


def full_rel(a, b, fp32=False):
    """Relative Frobenius difference of two device tensors holding the same
    data kind (real and imaginary parts alike; sums in FP64)."""
    import torch
    dt = torch.float32 if fp32 else torch.float64
    x, y = a.view(dt).double(), b.view(dt).double()
    return float(torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y))


def sig(x, n=4):
    """x rounded to n significant digits (keeps the bench line short)."""
    if x is None or x == 0 or x != x or x in (float("inf"), float("-inf")):
        return x
    from math import floor, log10
    return round(x, -int(floor(log10(abs(x)))) + (n - 1))


def ccsd_case(X, s, s_obj, name, steps, warmup, nsamp, psteps=None, world=1, on_timed=None, after_timed=None,
              on_warmup=None):
    """Chosen (METHOD_AUTO: the plan selector) against plain TTGT for one
    CCSD-like workload: device-timed TFLOP/s of both, the chosen D compared with
    the plain D over the WHOLE output tensor, and (R8/C8) both against the
    double-double oracle on `nsamp` sampled elements.  Returns the compact
    record, the device case and (chosen ms, plain ms, stats, timed-GEMM ms and
    count of the chosen steps, of the plain steps)."""
    import torch
    wl = WORKLOADS[name]
    case = ContractionCase(X, wl, s)
    case.run(X.METHOD_AUTO)  # first call of a shape: the selector may time close candidates
    torch.cuda.synchronize()
    if on_warmup:
        on_warmup()  # e.g. the clock sampler, started early so that it is running in the timed region
    X.timing_enable(True)  # CUDA events around the GEMM launches, read after each timed region

    def hook():
        X.timing_read()
        if on_timed:
            on_timed()
    ms = time_steps(lambda: case.run(X.METHOD_AUTO), steps, warmup, world, s_obj, on_timed=hook) / steps
    if after_timed:
        after_timed()
    gemm = X.timing_read()
    st = X.last_contract_stats()
    psteps = psteps or max(1, steps // 2)
    pms = time_steps(lambda: case.run(X.METHOD_TTGT), psteps, 1, world, s_obj,
                     on_timed=lambda: X.timing_read()) / psteps
    pgemm = X.timing_read()
    X.timing_enable(False)
    # whole-tensor comparison: plain D, then chosen D (both non-accumulating)
    case.run(X.METHOD_TTGT, accumulative=False)
    torch.cuda.synchronize()
    dplain = case.D.clone()
    err_p = sample_error(X, case, nsamp) if nsamp and wl["dtk"] in (8, 18) else None
    case.run(X.METHOD_AUTO, accumulative=False)
    torch.cuda.synchronize()
    err_c = sample_error(X, case, nsamp) if nsamp and wl["dtk"] in (8, 18) else None
    rel = full_rel(case.D, dplain, fp32=wl["dtk"] in (4, 14))
    case.dchosen = case.D.clone()
    del dplain
    rec = {"chosen": {"method": {1: "ttgt", 2: "fused"}.get(st.method, st.method), "moduli": st.moduli,
                      "slices": st.slices,
                      "tile_n": st.tile_n, "tile_m": st.tile_m, "ms": sig(ms), "TFLOP/s": sig(case.flops / ms / 1e9)},
           "plain": {"ms": sig(pms), "TFLOP/s": sig(case.flops / pms / 1e9)},
           "chosen_over_plain": sig(pms / ms, 3),
           "rel_frob_chosen_vs_plain_whole_D": sig(rel, 3)}
    if err_c:
        rec["dd_samples"] = {"n": nsamp, "chosen_rel_frob": sig(err_c["rel_frobenius"], 3),
                             "plain_rel_frob": sig(err_p["rel_frobenius"], 3),
                             "chosen_max_abs": sig(err_c["max_abs"], 3)}
    return rec, case, (ms, pms, st, gemm, pgemm)


def c1_case(X, s, s_obj):
    """The single-block 40^4 R8 configuration: D(a,b,c,d) += 0.5 *
    L(c,k,a,l) * R(l,d,k,b), L and R from one seeded stream (seed 0, L first),
    D = 0; chosen and plain rates, the error of both against the double-double
    oracle over the whole tensor, and the (3,1,4,2) permutation of L."""
    import numpy as np
    import torch

    import oracle as O
    pat, n = "D(a,b,c,d)+=L(c,k,a,l)*R(l,d,k,b)", 40
    dims, nvol = [n] * 4, n ** 4
    u = O.splitmix64_uniform(2 * nvol, 0)
    L, R = u[:nvol].copy(), u[nvol:].copy()
    ref = np.zeros(nvol)
    cptrn, *_ = O.parse_pattern(pat)
    O.contract(cptrn, ref, dims, L, dims, R, dims, 0.5, mode=1)
    dL, dR = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    dD = torch.zeros(nvol, dtype=torch.float64, device="cuda")
    out = {"workload": f"{pat} 40^4 R8 alpha 0.5, seed 0, D=0"}
    flops = 2.0 * 1600 ** 3
    for key, method in (("chosen", X.METHOD_AUTO), ("plain", X.METHOD_TTGT)):
        def run(acc=True, method=method):
            X.tensor_contract(pat, 8, dims, dD.data_ptr(), dims, dL.data_ptr(), dims, dR.data_ptr(), 0.5, 0, acc,
                              X.make_plan(method), s)
        run()
        ms = time_back_to_back(run, 20, s_obj) / 20
        dD.zero_()
        run()
        err = O.rel_frobenius(dD.cpu().numpy(), ref)
        out[key] = {"method": {1: "ttgt", 2: "fused"}.get(X.last_contract_stats().method), "ms": sig(ms),
                    "TFLOP/s": sig(flops / ms / 1e9), "rel_frob_vs_dd": sig(err, 3)}
    dP = torch.empty_like(dL)
    cp = lambda: X.tensor_copy(8, dims, (3, 1, 4, 2), dL.data_ptr(), dP.data_ptr(), 0, s)
    cp()
    pms = time_back_to_back(cp, 20, s_obj) / 20
    exact = bool(np.array_equal(dP.cpu().numpy(), O.permute(L, dims, [3, 1, 4, 2])))
    out["permute_3142"] = {"GB/s": sig(2.0 * nvol * 8 / pms / 1e6), "bit_exact_vs_oracle": exact}
    return out


# ----------------------------------------------------------------------- permutations
SWEEP_DIMS = {8: {2: [5793] * 2, 3: [322] * 3, 4: [76] * 4, 5: [32] * 5, 6: [18] * 6},
              4: {2: [8192] * 2, 3: [406] * 3, 4: [90] * 4, 5: [37] * 5, 6: [20] * 6}}
# skewed shapes: (rank, small extent, its position); the other extents are
# balanced to the governing 256 MiB volume
SKEWED = [(3, 3, 0), (3, 2, 2), (4, 5, 0), (4, 7, 3), (6, 2, 0), (6, 4, 5)]


def skewed_dims(dtk, rank, small, pos):
    target = 2 ** 25 if dtk == 8 else 2 ** 26
    rest = int(round((target / small) ** (1.0 / (rank - 1))))
    dims = [rest] * rank
    dims[pos] = small
    return dims


def sweep_cases():
    """The permutation sweep: 256 MiB-class R8 and R4 tensors of rank 2-6
    (extents in SWEEP_DIMS: all permutations at ranks 2-4, 24 seeded random
    ones at rank 5, 40 at rank 6) and skewed shapes (one extent of 2-7, six
    seeded permutations each, the reversal first).  Returns dicts with dtk,
    dims, perm and the class name ("r8_4", "r4_6", "r8_4s", ...)."""
    import itertools
    import random
    rng = random.Random(20240601)

    def random_perms(rank, n, first=()):
        perms = list(first)
        while len(perms) < n:
            p = list(range(1, rank + 1))
            rng.shuffle(p)
            if tuple(p) not in perms:
                perms.append(tuple(p))
        return perms
    out = []
    for dtk in (8, 4):
        tag = "r8" if dtk == 8 else "r4"
        for rank, dims in SWEEP_DIMS[dtk].items():
            perms = (list(itertools.permutations(range(1, rank + 1))) if rank <= 4
                     else random_perms(rank, 24 if rank == 5 else 40))
            out += [dict(dtk=dtk, dims=list(dims), perm=tuple(p), cls=f"{tag}_{rank}") for p in perms]
        for rank, small, pos in SKEWED:
            dims = skewed_dims(dtk, rank, small, pos)
            out += [dict(dtk=dtk, dims=dims, perm=p, cls=f"{tag}_{rank}s")
                    for p in random_perms(rank, 6, [tuple(range(rank, 0, -1))])]
    return out


# the configuration's own example extents, larger than the governing 256 MiB
# (128^4: 2 GiB in R8, 1 GiB in R4; 24^6: 1.4 GiB / 0.7 GiB): extra points
EXAMPLE_SHAPES = [(8, [128] * 4), (4, [128] * 4), (8, [24] * 6), (4, [24] * 6)]


def example_cases():
    """Four permutations of each example shape: at rank 4 the reversal, the
    slowest 256 MiB class's (4,3,1,2), (3,4,1,2) and (2,1,4,3); at rank 6 the
    reversal and three seeded random ones."""
    import random
    rng = random.Random(20240602)
    out = []
    for dtk, dims in EXAMPLE_SHAPES:
        r = len(dims)
        if r == 4:
            perms = [(4, 3, 2, 1), (4, 3, 1, 2), (3, 4, 1, 2), (2, 1, 4, 3)]
        else:
            perms = [tuple(range(r, 0, -1))]
            while len(perms) < 4:
                p = list(range(1, r + 1))
                rng.shuffle(p)
                if tuple(p) not in perms:
                    perms.append(tuple(p))
        tag = ("r8_" if dtk == 8 else "r4_") + "x".join(str(x) for x in dims[:1]) + f"^{r}"
        out += [dict(dtk=dtk, dims=list(dims), perm=p, cls=tag) for p in perms]
    return out


def add_cases():
    """The add sweep (D += 0.37 * permute(L)): all 24 rank-4 permutations and
    the first 10 rank-6 ones, R8 and R4, at the sweep's 256 MiB sizes."""
    cases = sweep_cases()
    out = [c for c in cases if c["cls"] in ("r8_4", "r4_4")]
    for tag in ("r8_6", "r4_6"):
        out += [c for c in cases if c["cls"] == tag][:10]
    return out


def torch_order(perm):
    """torch.permute order that applies the O2N permutation `perm` (input
    dimension i goes to output position perm[i]) to a dlf tensor viewed as a
    C-order torch tensor of reversed extents."""
    r = len(perm)
    q = [0] * r
    for i, p in enumerate(perm):
        q[p - 1] = i
    return [r - 1 - q[r - 1 - a] for a in range(r)]


def torch_permuted(t, dims, perm, word):
    """permute(t) computed by torch, as an independent check of the bits: t
    holds a dlf tensor of extents dims, viewed as words of dtype `word`."""
    x = t.view(word)
    if len(dims) > 1:
        x = x.view(*reversed(dims)).permute(*torch_order(perm)).contiguous()
    return x.view(-1)


def permute_sweep(X, stream, stream_obj, hbm_gbs, with_add=True, per_case=False, cases=None, examples=True):
    """Every sweep case: 10 back-to-back timed copies after the first call (where
    the library's measured plan choice runs), and a bit-for-bit comparison of
    the result with torch's permute of the same device data.  Per class the
    aggregate (bytes over time) and the slowest case, in GB/s; then the add
    sweep, and the example shapes as extra points."""
    import torch
    cases = sweep_cases() if cases is None else cases
    stats, rates, mism = {}, [], 0
    tot_b = tot_s = 0.0
    cur, a, b = None, None, None
    for c in cases:
        dtk, dims, perm = c["dtk"], c["dims"], c["perm"]
        es = X.ELEM_BYTES[dtk]
        nvol = vol(dims)
        if cur != (dtk, tuple(dims)):
            a = b = None
            torch.cuda.empty_cache()
            a = torch.empty(nvol * es, dtype=torch.uint8, device="cuda")
            b = torch.empty_like(a)
            X.fill_uniform(dtk, nvol, a.data_ptr(), 3, stream=stream)
            cur = (dtk, tuple(dims))
        fn = lambda: X.tensor_copy(dtk, dims, perm, a.data_ptr(), b.data_ptr(), 0, stream)
        fn()
        ms = time_back_to_back(fn, 10, stream_obj) / 10
        word = torch.int64 if es == 8 else torch.int32
        if not torch.equal(b.view(word), torch_permuted(a, dims, perm, word)):
            mism += 1
        gb = 2.0 * nvol * es / 1e9
        rates.append(gb / (ms / 1e3))
        tot_b += gb
        tot_s += ms / 1e3
        st = stats.setdefault(c["cls"], [0.0, 0.0, 1e30])
        st[0] += gb
        st[1] += ms / 1e3
        st[2] = min(st[2], gb / (ms / 1e3))
    a = b = None
    agg = tot_b / tot_s
    r4 = [(2.0 * vol(c["dims"]) * X.ELEM_BYTES[c["dtk"]] / 1e9, r) for c, r in zip(cases, rates)
          if c["cls"] in ("r8_4", "r4_4")] or [(1.0, agg)]
    out = {"GB/s": round(agg, 1), "min_GB/s": round(min(rates), 1), "frac_measured_hbm": sig(agg / hbm_gbs, 3),
           "frac_8000": sig(agg / 8000.0, 3), "min_frac_measured_hbm": sig(min(rates) / hbm_gbs, 3),
           "cases": len(cases), "bit_exact": len(cases) - mism,
           "rank4_48": {"GB/s": round(sum(g for g, _ in r4) / sum(g / r for g, r in r4), 1),
                        "min": round(min(r for _, r in r4), 1)},
           "by_class_agg_min": {k: [round(v[0] / v[1]), round(v[2])] for k, v in stats.items()}}
    if per_case:
        out["per_case"] = [[c["cls"], c["dims"], list(c["perm"]), round(r)] for c, r in zip(cases, rates)]
    if with_add:
        out["add"] = add_sweep(X, stream, stream_obj, hbm_gbs, per_case=per_case)
    if examples:
        try:
            ex = permute_sweep(X, stream, stream_obj, hbm_gbs, with_add=False, per_case=per_case,
                               cases=example_cases(), examples=False)
            out["examples"] = {k: ex[k] for k in ("GB/s", "min_GB/s", "cases", "bit_exact", "by_class_agg_min")}
            if per_case:
                out["examples"]["per_case"] = ex["per_case"]
        except Exception as exc:  # reported, not fatal
            out["examples"] = {"error": str(exc)[:200]}
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
    out["timing"] = "10 back-to-back calls per case after the first; bits checked against torch.permute"
    return out


def add_sweep(X, stream, stream_obj, hbm_gbs, scale=0.37, per_case=False):
    """D += scale * permute(L) over add_cases(): 3 * vol * elem bytes per call;
    one call per case from a fresh D compared bit for bit with torch's
    d + permute(l) * scale (two roundings), then 10 back-to-back timed calls."""
    import torch
    cases = add_cases()
    cur, tot_b, tot_s, rates, mism = None, 0.0, 0.0, [], 0
    l = d0 = d = None
    for c in cases:
        dtk, dims, perm = c["dtk"], c["dims"], c["perm"]
        es = X.ELEM_BYTES[dtk]
        nvol = vol(dims)
        if cur != (dtk, tuple(dims)):
            l = d0 = d = None
            torch.cuda.empty_cache()
            l = torch.empty(nvol * es, dtype=torch.uint8, device="cuda")
            d0 = torch.empty_like(l)
            d = torch.empty_like(l)
            X.fill_uniform(dtk, nvol, l.data_ptr(), 4, stream=stream)
            X.fill_uniform(dtk, nvol, d0.data_ptr(), 5, stream=stream)
            cur = (dtk, tuple(dims))
        fdt = torch.float64 if es == 8 else torch.float32
        d.copy_(d0)
        X.tensor_add(dtk, dims, perm, d.data_ptr(), l.data_ptr(), scale, 0, stream)
        ref = d0.view(fdt) + torch_permuted(l, dims, perm, fdt) * scale
        if not torch.equal(d.view(torch.uint8), ref.view(torch.uint8)):
            mism += 1
        fn = lambda: X.tensor_add(dtk, dims, perm, d.data_ptr(), l.data_ptr(), scale, 0, stream)
        ms = time_back_to_back(fn, 10, stream_obj) / 10
        gb = 3.0 * nvol * es / 1e9
        rates.append(gb / (ms / 1e3))
        tot_b += gb
        tot_s += ms / 1e3
    l = d0 = d = None
    agg = tot_b / tot_s
    out = {"GB/s": round(agg, 1), "min_GB/s": round(min(rates), 1), "frac_measured_hbm": sig(agg / hbm_gbs, 3),
           "cases": len(cases), "bit_exact": len(cases) - mism}
    if per_case:
        out["per_case"] = [[c["cls"], c["dims"], list(c["perm"]), round(r)] for c, r in zip(cases, rates)]
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
    library's CUDA kernels on the first 80% of the corpus, evaluated on the rest
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
    if T.shape[1] != len(S.PLANS):
        return None  # a corpus of another plan space
    # the first 16000 entries train, the last 4000 are held out (rows without
    # a label for a plan that applies to every data kind are left out of both)
    always = [i for i in range(T.shape[1]) if i not in S.FP64_ONLY]
    ok = np.isfinite(T[:, always]).all(axis=1)
    split = int(0.8 * len(F))
    n_train = int(ok[:split].sum())
    F, T = F[ok], T[ok]
    t0 = time.perf_counter()
    params, mean, scale, hist = S.train(F[:n_train], T[:n_train], hidden=128, epochs=150, seed=0, log_every=149)
    train_s = time.perf_counter() - t0
    pred = S.predict(params, mean, scale, F[n_train:], hidden=128)
    learned = S.evaluate(T[n_train:], S.choose(pred, F[n_train:]))
    rule = S.evaluate(T[n_train:], [S.rule_choice(f) for f in F[n_train:]])
    always = {name: S.evaluate(T[n_train:], [i] * (len(F) - n_train))["total_time_regret"]
              for i, name in enumerate(S.PLAN_NAMES) if i not in S.FP64_ONLY}
    X.selector_install(128, params, mean, scale)
    t0 = time.perf_counter()
    for f in F[n_train:n_train + 2000]:
        X.selector_choose(f)
    host_us = (time.perf_counter() - t0) / min(2000, len(F) - n_train) * 1e6
    lib_us = float(np.median([X.selector_time(f, 2000) for f in F[n_train:n_train + 16]]))
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
    return {"corpus": f"{len(ok)} random contractions (seed 0), {int(ok.sum())} with every plan labelled: "
                      f"{n_train} of the first {split} train, {len(F) - n_train} of the last {len(ok) - split} "
                      f"held out", "plans": S.PLAN_NAMES,
            "learned": learned, "size_rule": rule, "always_one_plan_total_regret": always,
            "train_seconds": round(train_s, 1), "final_train_loss": round(hist[-1][1], 4) if hist else None,
            "selection_us_library": round(lib_us, 3), "selection_us_python": round(host_us, 2),
            "selection_us_gpu_batched": round(gpu_us, 4)}


def e2e_talsh(X, wl, steps, case=None):
    """The same contraction through talshTensorContract (the reference-facing
    API) with Host-resident tensors: every call copies V, T and D to the GPU
    and D back (copy control TTT).  The host tensors hold the device case's
    seeded data; after the calls D / (number of calls) is compared with the
    device result of the chosen method over the whole tensor."""
    import numpy as np
    import torch

    import exatensor_b200.talsh as T
    T.init((int(os.environ.get("LOCAL_RANK", "0")),))
    dd, ld, rd = shapes(wl["pattern"], wl["v"], wl["o"])
    es = X.ELEM_BYTES[wl["dtk"]]
    D = T.Tensor(dd, wl["dtk"], 0.0)
    L = T.Tensor(ld, wl["dtk"], 0.0)
    R = T.Tensor(rd, wl["dtk"], 0.0)
    seeded = case is not None
    if seeded:
        for t, src in ((L, case.L), (R, case.R)):
            torch.from_numpy(t.host_array().view(np.uint8)).copy_(src)
        torch.cuda.synchronize()
    run = lambda: T.check(T.contract(wl["pattern"], D, L, R, 1.0, 0, T.DEV_NVIDIA_GPU, T.COPY_TTT, True),
                          "talshTensorContract")
    for _ in range(2):  # the second call of a shape may time close plan candidates once
        run()
    t0 = time.perf_counter()
    for _ in range(steps):
        run()
    dt = (time.perf_counter() - t0) / steps
    flops = 2.0 * vol(dd) * (vol(ld) * vol(rd) / vol(dd)) ** 0.5
    res = {"value": sig(flops / dt / 1e12), "unit": "TFLOP/s", "ms_per_step": sig(dt * 1e3),
           "h2d_bytes_per_step": (vol(dd) + vol(ld) + vol(rd)) * es, "d2h_bytes_per_step": vol(dd) * es,
           "api": "talshTensorContract(COPY_TTT), host tensors, wall clock incl. H2D/D2H",
           "path": ("inputs streamed to the GPU in slices under the computation" if os.environ.get("TB_STREAM") != "0"
                    else "inputs staged whole, then the contraction")}
    # PCIe ceiling: pinned host <-> device copies of 1 GiB, CUDA events
    hb = torch.empty(1 << 30, dtype=torch.uint8, pin_memory=True)
    db = torch.empty(1 << 30, dtype=torch.uint8, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    bw = {}
    for name, fn in (("h2d", lambda: db.copy_(hb, non_blocking=True)), ("d2h", lambda: hb.copy_(db, non_blocking=True))):
        fn()
        e0.record()
        for _ in range(3):
            fn()
        e1.record()
        e1.synchronize()
        bw[name] = 3 * (1 << 30) / (e0.elapsed_time(e1) / 1e3) / 1e9
    del hb, db
    xfer_ms = (res["h2d_bytes_per_step"] / bw["h2d"] + res["d2h_bytes_per_step"] / bw["d2h"]) / 1e6
    res["pcie"] = {"h2d_gbs": sig(bw["h2d"]), "d2h_gbs": sig(bw["d2h"]), "transfer_ms_per_step": sig(xfer_ms),
                   "transfer_frac_of_step": sig(xfer_ms / (dt * 1e3), 3),
                   "how": "pinned 1 GiB copies, CUDA events; transfer_ms = H2D bytes / H2D rate + D2H bytes / D2H rate"}
    if seeded and getattr(case, "dchosen", None) is not None:
        got = torch.from_numpy(D.host_array().copy()).cuda() / float(2 + steps)
        res["rel_frob_vs_device_result"] = sig(full_rel(got.view(torch.uint8), case.dchosen), 3)
        del got
    del D, L, R
    return res


def measure_peaks(X, s):
    """Tensor-core rates of this GPU from the library's own probes
    (tb_peak_measure: operands on chip, no DRAM traffic), in T(FL)OP/s: INT8
    tcgen05 as a burst (one ~20 ms launch) and sustained (~1.5 s at the power
    cap), BF16 tcgen05 (burst; compare with the cuBLAS figure in
    MEASURED_PEAKS.json) and FP64 DMMA."""
    i8, _ = X.peak_measure(X.PEAK_I8, 280000, s)
    i8s, i8s_ms = X.peak_measure(X.PEAK_I8, 14000000, s)
    bf, _ = X.peak_measure(X.PEAK_BF16, 280000, s)
    f64, _ = X.peak_measure(X.PEAK_F64, 60000, s)
    return {"i8_tops_burst": sig(i8 / 1e12), "i8_tops_sustained": sig(i8s / 1e12), "sustained_ms": sig(i8s_ms),
            "bf16_tflops_burst": sig(bf / 1e12), "f64_tflops": sig(f64 / 1e12),
            "how": "tb_peak_measure: back-to-back MMAs on shared-memory operands, one CTA per SM (DMMA: 4 chains "
                   "per warp), CUDA events"}


# ----------------------------------------------------------------------------- CPU
CPU_SAMPLE_A = 48  # the CPU legs contract rows a < 48 of the v=192 workload (1/4 of its FLOPs)


def cpu_contraction_sample(steps=1, warmup=1, workload="ccsd1_r8"):
    """The reference's OpenMP+BLAS CPU contraction path (restated in oracle/:
    cache-blocked OpenMP permutes and OpenBLAS dgemm, as tensor_block_contract
    runs them) on a bounded sample of the headline workload: the output rows
    a < 48 of the v=192 contraction, i.e. the same pattern with the extent of
    a cut to 48 (M = 9216 of 36864, N and K as in the full workload).
    Returns the mean over `steps` timed calls after `warmup` untimed ones."""
    import numpy as np

    import oracle as O
    nthr = O.nthreads_default()
    if not O.blas_available():
        return None
    wl = WORKLOADS[workload]
    dd, ld, rd = shapes(wl["pattern"], wl["v"], wl["o"])
    dd[0], ld[0] = CPU_SAMPLE_A, CPU_SAMPLE_A  # a is the first index of D and of V
    cptrn, *_ = O.parse_pattern(wl["pattern"])
    L = O.fill_uniform(vol(ld), 1) / wl["v"]
    R = O.fill_uniform(vol(rd), 2)
    D = np.zeros(vol(dd))
    for _ in range(max(0, warmup)):
        O.contract_blas(cptrn, D, dd, L, ld, R, rd, 1.0, True, nthr)
    times = []
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        O.contract_blas(cptrn, D, dd, L, ld, R, rd, 1.0, True, nthr)
        times.append(time.perf_counter() - t0)
    flops = 2.0 * vol(dd) * (vol(ld) * vol(rd) / vol(dd)) ** 0.5
    mean = sum(times) / len(times)
    return {"value": sig(flops / mean / 1e12), "unit": "TFLOP/s", "cores": nthr, "kind": "port",
            "ms_per_step": sig(mean * 1e3),
            "sample": f"rows a<{CPU_SAMPLE_A} of the v={wl['v']} workload ({flops:.3e} FLOP per step, 1/4 of it): "
                      f"OpenMP blocked permutes + OpenBLAS dgemm, mean of {len(times)} after {max(0, warmup)}"}


def config_of(name):
    """The bench line's config, identical in both arms."""
    wl = WORKLOADS[name]
    return {"workload": f"{name}: {wl['pattern']} v={wl['v']} o={wl['o']}",
            "l2": "inputs larger than L2 (V alone is 10.9 GB in R8)"}


DATA = "synthetic (seeded splitmix64 U[-1,1), V scaled 1/v, D=0)"


def run_reference(args):
    """Reference arm: the reference's CPU implementation of the path (its
    OpenMP+BLAS CP-TAL contraction, restated in oracle/ because the Fortran
    reference cannot be compiled here), on this host's cores, rank 0 only."""
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import oracle as O
    O.build()
    res = cpu_contraction_sample(steps=max(1, args.steps), warmup=args.warmup, workload=args.workload)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "bundled OpenBLAS not found"}))
        return
    line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": "TFLOP/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": {4: "f32", 8: "f64"}[WORKLOADS[args.workload]["dtk"]],
            "data": DATA, "config": config_of(args.workload), "cpu_baseline": res,
            "e2e": {"value": res["value"], "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ----------------------------------------------------------------------------- main
OTHER_CONFIGS = ["ccsd2_r8", "ccsd1_c8", "ccsd2_c8", "ccsd1_r4", "ccsd2_r4"]


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
    extras = world == 1 and not args.headline_only  # the rest of the line runs on one GPU only
    pk = measure_peaks(X, s) if rank == 0 else None
    bsc = None
    if extras and not args.no_block_sparse:
        try:
            bsc = block_sparse_case(X, s, s_obj, 8, steps=1)
        except Exception as exc:  # reported, not fatal: the headline contraction still runs
            bsc = {"error": str(exc)[:300]}
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
    clocks = Clocks(local)
    cnt = {}

    def start():
        cnt["n0"] = X.launch_count()

    def stop():
        cnt["clk"] = clocks.stop()
        cnt["launches"] = X.launch_count() - cnt["n0"]
    rec, case, (ms, pms, st, gemm, pgemm) = ccsd_case(
        X, s, s_obj, args.workload, args.steps, args.warmup, nsamp=4096 if rank == 0 else 0,
        psteps=max(1, args.steps // 2), world=world, on_timed=start, after_timed=stop, on_warmup=clocks.start)
    ms_max = max_over_ranks(ms, world)
    pms_max = max_over_ranks(pms, world)
    value = world * case.flops / (ms_max / 1e3) / 1e12
    plain = case.flops / (pms_max / 1e3) / 1e12
    chosen_method = {1: "ttgt", 2: "fused"}.get(st.method, str(st.method))
    line = None
    if rank == 0:
        gemm_ms, gemm_n = gemm
        per_launch_ms = gemm_ms / max(1, gemm_n)
        i8 = wl["dtk"] in (8, 18)
        if chosen_method == "fused":
            kern = ("tc_gemm_kernel: tcgen05 INT8 GEMM, " + (f"{st.moduli} modular residues" if st.moduli
                                                                else f"{st.slices} slices")) if i8 else \
                "tc_gemm_kernel: tcgen05 split-BF16 GEMM"
            hw_ops = case.flops * max(1, st.products)  # each slice pair / BF16 term is a full GEMM
            peak = pk["i8_tops_sustained"] if i8 else bf16_tflops
            peak_note = ("measured: tb_peak_measure INT8 tcgen05, sustained (the GEMM runs back to back for the "
                         "whole timed region)" if i8 else f"{peak_src} cuBLAS bf16 burst (MEASURED_PEAKS.json)")
        else:
            kern = "dgemm_tn_kernel: FP64 DMMA" if i8 else "sgemm_tn_kernel: FP32 FFMA"
            hw_ops = case.flops
            peak = pk["f64_tflops"]
            peak_note = "measured: tb_peak_measure FP64 DMMA"
        achieved = hw_ops / (per_launch_ms / 1e3) / 1e12 if gemm_n else None
        roofline = {"bound": "tensor", "kernel": kern, "achieved": sig(achieved) if achieved else None,
                    "peak": peak, "unit": "TFLOP/s", "frac": sig(achieved / peak, 3) if achieved else None,
                    "traffic": TC_GEMM_TRAFFIC if (chosen_method == "fused" and args.workload == "ccsd1_r8") else None,
                    "traffic_note": "dram read+write bytes per launch (ncu, v=96 case scaled by the 16x work)",
                    "peak_source": peak_note, "frac_of_burst": sig(achieved / pk["i8_tops_burst"], 3)
                    if (achieved and chosen_method == "fused" and i8) else None,
                    "launch_ms": sig(per_launch_ms), "launches_timed": gemm_n}
        plain_rec = {"value": sig(plain), "unit": "TFLOP/s", "method": "ttgt: permute + FP64 DMMA GEMM + permute",
                     "gemm_ms_per_launch": sig(pgemm[0] / max(1, pgemm[1])),
                     "gemm_frac_of_measured_f64": sig(case.flops / (pgemm[0] / max(1, pgemm[1]) / 1e3) / 1e12
                                                      / pk["f64_tflops"], 3) if pgemm[1] else None}
        error = {"chosen_vs_plain_whole_D_rel_frob": rec["rel_frob_chosen_vs_plain_whole_D"],
                 "dd_samples": rec.get("dd_samples"), "bound": 1e-12}
        e2e = configs = c1 = perm = sel = cpu = None
        if extras:
            e2e = e2e_talsh(X, wl, steps=max(1, min(2, args.steps)), case=case)
        del case
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        if extras:
            configs = {}
            for name in OTHER_CONFIGS:
                try:
                    r, c, _ = ccsd_case(X, s, s_obj, name, 3, 1, nsamp=256, psteps=1)
                    configs[name] = r
                    del c
                except Exception as exc:  # reported, not fatal
                    configs[name] = {"error": str(exc)[:200]}
                torch.cuda.synchronize()
                torch.cuda.empty_cache()
            c1 = c1_case(X, s, s_obj)
            perm = permute_sweep(X, s, s_obj, hbm_gbs)
            try:
                sel = selector_case(X)
            except Exception as exc:  # reported, not fatal
                sel = {"error": str(exc)[:300]}
            cpu = cpu_contraction_sample(steps=3, warmup=1)
        if e2e is None:
            e2e = {"value": None, "note": "end-to-end leg runs at N=1"}
        line = {
            "metric": METRIC, "value": sig(value, 5), "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sig(ms_max, 5), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {4: "f32", 8: "f64", 14: "c64", 18: "c128"}[wl["dtk"]], "data": DATA,
            "config": config_of(args.workload),
            "permute": perm, "configs": configs, "c1": c1, "block_sparse": bsc, "selector": sel, "peaks": pk,
            "plan": {"method": chosen_method, "moduli": st.moduli, "residue_bits": st.residue_bits,
                     "slices": st.slices, "passes": st.passes, "products": st.products,
                     "tile_n": st.tile_n, "tile_m": st.tile_m, "parallelism": f"replicas x{world}"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": cnt.get("clk"),
            "gpu_launches": cnt.get("launches"),
            "plain": plain_rec, "chosen_over_plain": sig(value / world / plain, 3), "error": error,
        }
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line, separators=(",", ":")))


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
        for name in names:
            rec, c, _ = ccsd_case(X, s, s_obj, name, max(1, args.steps), max(1, args.warmup), nsamp=256, psteps=1)
            print(json.dumps({"profile": "configs", "workload": name, **rec}), flush=True)
            del c
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
        return
    if args.profile == "sweep":
        print(json.dumps({"profile": "sweep", **permute_sweep(X, s, s_obj, peaks()[0], per_case=True)}))
        return
    if args.profile == "examples":
        print(json.dumps({"profile": "examples", **permute_sweep(X, s, s_obj, peaks()[0], with_add=False, per_case=True,
                                                                 cases=example_cases(), examples=False)}))
        return
    if args.profile == "peaks":
        print(json.dumps({"profile": "peaks", **measure_peaks(X, s)}))
        return
    if args.profile == "c1":
        print(json.dumps({"profile": "c1", **c1_case(X, s, s_obj)}))
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
    if args.profile == "permute" and args.case:
        # one case, e.g. --case 4:37x37x37x37x37:1,3,5,4,2 (data kind : extents : O2N permutation)
        k, dstr, pstr = args.case.split(":")
        dtk, dims, perm = int(k), [int(x) for x in dstr.split("x")], [int(x) for x in pstr.split(",")]
        es = X.ELEM_BYTES[dtk]
        v = vol(dims)
        a = torch.empty(v * es, dtype=torch.uint8, device="cuda")
        b = torch.empty_like(a)
        X.fill_uniform(dtk, v, a.data_ptr(), 3, stream=s)
        ms = time_steps(lambda: X.tensor_copy(dtk, dims, perm, a.data_ptr(), b.data_ptr(), 0, s), args.steps,
                        args.warmup, 1, s_obj)
        print(json.dumps({"profile": "permute", "case": args.case,
                          "GB/s": round(2.0 * v * es * args.steps / (ms / 1e3) / 1e9, 1)}))
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
                      "method": st.method, "moduli": st.moduli, "slices": st.slices, "products": st.products,
                      "tile_n": st.tile_n,
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
    ap.add_argument("--headline-only", action="store_true",
                    help="only the headline contraction (no sweep, configs, selector, e2e or CPU legs)")
    ap.add_argument("--profile", choices=["contract", "plain", "permute", "permsweep", "bsc", "selector", "e2e",
                                          "configs", "sweep", "examples", "peaks", "c1"],
                    default=None,
                    help="run one part on a small case for a profiler (no bench line)")
    ap.add_argument("--case", default=None, help="--profile permute: one case, data kind:extents:permutation")
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
