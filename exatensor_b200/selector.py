"""Learned plan selection for tensor contractions.

A small MLP maps a contraction descriptor (sizes, ranks, index-map features,
data kind) to the predicted log-runtime of every candidate plan; the plan with
the smallest prediction is chosen.  The network is trained and evaluated by
the library's own CUDA kernels (``tb_mlp_*`` in ``libtalsh_b200.so``) on
timings that the autotuner records for a seeded corpus of random contractions.
It only chooses among plans that all meet the accuracy bounds, so it never
changes what a contraction computes beyond those bounds.

The random contractions follow the recipe of the reference's
``contr_pattern_rnd`` (TALSH/tensor_algebra_cpu.F90:5958): random operand
ranks, a random number of contracted indices placed at random positions of
both operands, and a random order of the uncontracted indices in the result.
"""
from __future__ import annotations

import math
import string

import numpy as np

# Candidate plans (make_plan arguments), in the order of the network's outputs
# and of the library's candidates (TB_SELECT_PLANS).  All of them meet the
# accuracy bounds; the INT8-slice plan applies to FP64 data only.
PLANS = [dict(method=1),                              # TTGT
         dict(method=2, tile_n=128),                  # tensor cores, 128-wide N tile
         dict(method=2, tile_n=256),                  # 256-wide N tile
         dict(method=2, tile_n=256, tile_m=256),      # 256-wide tile on SM pairs
         dict(method=2, tile_n=256, slices=6)]        # 6 INT8 slices instead of residues
PLAN_NAMES = ["ttgt", "fused_n128", "fused_n256", "fused_n256_pair", "fused_n256_slices6"]
FP64_ONLY = {4}
NFEAT = 16


def random_contraction(rng, max_rank=6, lo=2, hi=512, max_bytes=4 << 30, dtk=None):
    """One random contraction: (pattern, ddims, ldims, rdims, dtk)."""
    while True:
        lr = int(rng.integers(2, max_rank + 1))
        rr = int(rng.integers(2, max_rank + 1))
        nc = int(rng.integers(1, min(4, lr, rr) + 1))
        dr = lr + rr - 2 * nc
        if dr < 1 or dr > max_rank:
            continue
        labels = list(string.ascii_lowercase[: lr + rr - nc])
        contracted = labels[:nc]
        lfree = labels[nc: nc + lr - nc]
        rfree = labels[nc + lr - nc:]
        lidx = contracted + lfree
        ridx = contracted + rfree
        rng.shuffle(lidx)
        rng.shuffle(ridx)
        didx = lfree + rfree
        rng.shuffle(didx)
        ext = {x: int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))))) for x in labels}
        kind = dtk if dtk is not None else int(rng.choice([4, 8]))
        es = 8 if kind == 8 else 4
        vol = lambda idx: int(np.prod([ext[x] for x in idx])) if idx else 1
        # shrink the largest extents until the three operands fit the footprint cap
        while (vol(didx) + vol(lidx) + vol(ridx)) * es > max_bytes:
            big = max(labels, key=lambda x: ext[x])
            ext[big] = max(lo, ext[big] // 2)
        pattern = f"D({','.join(didx)})+=L({','.join(lidx)})*R({','.join(ridx)})"
        return pattern, [ext[x] for x in didx], [ext[x] for x in lidx], [ext[x] for x in ridx], kind


def rule_choice(desc):
    """The library's rule-based choice (select_method) as a plan index."""
    M, N, K = 2 ** desc[0], 2 ** desc[1], 2 ** desc[2]
    fused = M >= 64 and N >= 32 and K >= 64 and 2 * M * N * K >= 4e9
    if not fused:
        return 0
    return 2 if N >= 192 else 1


def choose(pred, features):
    """Plan with the smallest prediction among those the descriptor allows
    (the library's rule: INT8 slices for FP64 only)."""
    p = np.array(pred, dtype=np.float64, copy=True)
    fp64 = np.asarray(features)[..., 15] != 0
    for i in FP64_ONLY:
        p[..., i] = np.where(fp64, p[..., i], np.inf)
    return p.argmin(axis=-1)


def regret(times, choice):
    """Mean relative slowdown of the chosen plans against the best plan
    (plans without a label, NaN, do not count as best)."""
    t = np.asarray(times, dtype=np.float64)
    best = np.nanmin(t, axis=1)
    got = t[np.arange(len(t)), np.asarray(choice)]
    return float(np.mean(got / best - 1.0)), float(got.sum() / best.sum() - 1.0)


# ----------------------------------------------------------------------------- corpus labelling (GPU)
def label_corpus(n, seed=0, out=None, reps=2, log=None, start=0, long_ms=25.0, ttgt_long_ms=100.0):
    """Times every candidate plan of n seeded random contractions on the GPU.

    Returns (features [n][NFEAT], log-times [n][len(PLANS)] in ln(ms), NaN where
    a plan failed or does not apply, patterns).  Inputs are seeded uniform data
    in one buffer sized for the 4 GiB footprint cap.  Each plan's first run is
    timed between CUDA events on the launching stream; when it takes long_ms or
    more its time is the label (first-use costs are small beside it), else reps
    more runs are timed and their mean is the label.  TTGT's first run of a
    shape also chooses its permutation plans: it is the label only from
    ttgt_long_ms on, else a second run is timed (and reps more below
    long_ms).  A plan that fails, or leaves an error in the device error
    word, gets NaN."""
    import time

    import torch

    import exatensor_b200 as X
    X.device_init(0)
    s_obj = torch.cuda.current_stream()
    s = s_obj.cuda_stream
    # one input buffer per element type, each filled with finite values of its
    # own type (FP64 bit patterns read as FP32 would hold NaNs and infinities,
    # whose fix-up pass is not what the plans should be timed on); D goes to a
    # buffer of its own, so the inputs keep their values from one entry to the next
    cap = (4 << 30) + (1 << 20)
    bufs = {}
    for kind in (4, 8):
        bufs[kind] = torch.empty(cap, dtype=torch.uint8, device="cuda")
        X.fill_uniform(kind, cap // (8 if kind == 8 else 4), bufs[kind].data_ptr(), 1234, stream=s)
    dbuf = torch.empty(cap, dtype=torch.uint8, device="cuda")
    rng = np.random.default_rng(seed)
    feats, times, pats = [], [], []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_start = time.time()

    def timed(run, k):
        e0.record(s_obj)
        for _ in range(k):
            run()
        e1.record(s_obj)
        e1.synchronize()
        return e0.elapsed_time(e1) / k

    for i in range(n):
        pattern, dd, ld, rd, dtk = random_contraction(rng)
        if i < start:
            continue
        es = 8 if dtk == 8 else 4
        vol = lambda d: int(np.prod(d)) if d else 1
        lo = 0
        ro = (vol(ld) * es + 255) // 256 * 256
        base = bufs[8 if dtk == 8 else 4].data_ptr()
        dptr = dbuf.data_ptr()
        row = []
        for j, kw in enumerate(PLANS):
            if j in FP64_ONLY and dtk != 8:
                row.append(float("nan"))
                continue
            plan = X.make_plan(**kw)
            run = lambda: X.tensor_contract(pattern, dtk, dd, dptr, ld, base + lo, rd, base + ro, 1.0,
                                            accumulative=False, plan=plan, stream=s)
            try:
                t = timed(run, 1)
                if kw["method"] == 1 and t < ttgt_long_ms:
                    t = timed(run, 1)
                if t < long_ms:
                    t = timed(run, reps)
                X.device_check(s)
                row.append(math.log(max(t, 1e-4)))
            except X.TBError:
                torch.cuda.synchronize()
                row.append(float("nan"))
        feats.append(X.contract_descriptor(pattern, dtk, dd, ld, rd))
        times.append(row)
        pats.append(pattern + f" | {dd} {ld} {rd} dtk={dtk}")
        if out and ((i + 1) % 250 == 0 or i + 1 == n):
            np.savez_compressed(out, features=np.array(feats, np.float32), log_ms=np.array(times, np.float32),
                                patterns=np.array(pats), seed=seed, start=start)
            if log:
                print(f"{i + 1}/{n} labelled, {time.time() - t_start:.0f} s", file=log, flush=True)
    return np.array(feats, np.float32), np.array(times, np.float32), pats


# ----------------------------------------------------------------------------- training (GPU kernels)
def train(Xf, Y, hidden=128, epochs=200, batch=256, lr=2e-3, seed=0, log_every=0):
    """Trains the selector network with the library's CUDA kernels.

    Xf: [n][NFEAT] descriptors, Y: [n][len(PLANS)] ln(ms) (NaN = no label).
    Returns (params, mean, scale, loss history)."""
    import torch

    import exatensor_b200 as X
    Xf = np.asarray(Xf, np.float32)
    Y = np.asarray(Y, np.float32)
    mean = Xf.mean(axis=0)
    scale = Xf.std(axis=0)
    scale[scale < 1e-6] = 1.0
    Xn = (Xf - mean) / scale
    net = X.MLP(Xf.shape[1], hidden, Y.shape[1], max_batch=batch, seed=seed + 1)
    dev_x = torch.from_numpy(Xn).cuda()
    dev_y = torch.from_numpy(Y).cuda()
    rng = np.random.default_rng(seed)
    n = len(Xn)
    hist = []
    s = torch.cuda.current_stream().cuda_stream
    for ep in range(epochs):
        perm = torch.from_numpy(rng.permutation(n)).cuda()
        xs, ys = dev_x[perm].contiguous(), dev_y[perm].contiguous()
        tot = 0.0
        nb = 0
        for b0 in range(0, n - batch + 1, batch):
            want = log_every and (ep % log_every == 0 or ep == epochs - 1)
            loss = net.backward(xs[b0:b0 + batch].data_ptr(), ys[b0:b0 + batch].data_ptr(), batch, stream=s,
                                want_loss=bool(want))
            net.adam(lr=lr, stream=s)
            if want:
                tot += loss
                nb += 1
        if nb:
            hist.append((ep, tot / nb))
    params = net.params()
    net.close()
    return params, mean, scale, hist


def predict(params, mean, scale, Xf, hidden=128):
    """Predicted ln(ms) of every plan (GPU inference kernel)."""
    import torch

    import exatensor_b200 as X
    Xn = ((np.asarray(Xf, np.float32) - mean) / scale).astype(np.float32)
    nin = Xn.shape[1]
    # outputs from the parameter count: nin*h + h + h*h + h + h*o + o
    n_out = (len(params) - nin * hidden - 2 * hidden - hidden * hidden) // (hidden + 1)
    net = X.MLP(nin, hidden, n_out, max_batch=1024)
    net.set_params(params)
    dx = torch.from_numpy(Xn).cuda()
    dy = torch.empty((len(Xn), n_out), dtype=torch.float32, device="cuda")
    net.forward(dx.data_ptr(), len(Xn), dy.data_ptr())
    torch.cuda.synchronize()
    out = dy.cpu().numpy()
    net.close()
    return out


def evaluate(log_ms, choice):
    """Regret of plan choices against the best measured plan.  Rows need a
    label for every plan that applies to all data kinds; the FP64-only plan's
    label is NaN for FP32 rows and then does not count."""
    t = np.exp(np.asarray(log_ms, np.float64))
    always = [i for i in range(t.shape[1]) if i not in FP64_ONLY]
    ok = np.isfinite(t[:, always]).all(axis=1)
    t = t[ok]
    c = np.asarray(choice)[ok]
    if not np.all(np.isfinite(t[np.arange(len(t)), c])):
        raise ValueError("a plan was chosen that has no label")
    mean_regret, total_regret = regret(t, c)
    return {"rows": int(ok.sum()), "mean_regret": mean_regret, "total_time_regret": total_regret,
            "picked_best": float(np.mean(c == np.nanargmin(t, axis=1)))}


def save_weights(path, params, mean, scale, hidden=128, margin=0.0, autotune=0):
    """Writes a weights file for tb_selector_load / automatic loading."""
    import struct
    with open(path, "wb") as f:
        f.write(b"TBSEL001")
        f.write(struct.pack("<iiifi", NFEAT, hidden, len(PLANS), float(margin), int(autotune)))
        f.write(np.asarray(mean, "<f4").tobytes())
        f.write(np.asarray(scale, "<f4").tobytes())
        f.write(np.asarray(params, "<f4").tobytes())


def main(argv=None):
    import argparse
    import sys
    ap = argparse.ArgumentParser(description="selector corpus labelling and training")
    ap.add_argument("cmd", choices=["label", "train", "merge"])
    ap.add_argument("--parts", nargs="*", default=[], help="merge: chunk files written by label --start")
    ap.add_argument("--corpus", default=None, help="train: labelled corpus (.npz)")
    ap.add_argument("--epochs", type=int, default=150)
    ap.add_argument("--margin", type=float, default=0.25, help="train: ln-time margin below which AUTO times plans")
    ap.add_argument("--autotune", type=int, default=1)
    ap.add_argument("--n", type=int, default=20000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--start", type=int, default=0)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--out", required=True, help="label: corpus .npz; train: weights file")
    a = ap.parse_args(argv)
    if a.cmd == "label":
        label_corpus(a.n, a.seed, a.out, reps=a.reps, log=sys.stdout, start=a.start)
        return
    if a.cmd == "merge":
        # chunks of one seeded sequence, each starting where the previous ended
        parts = sorted((np.load(p) for p in a.parts), key=lambda d: int(d["start"]))
        nxt = 0
        for d in parts:
            if int(d["start"]) != nxt:
                raise SystemExit(f"chunk starting at {int(d['start'])} does not follow entry {nxt}")
            nxt += len(d["features"])
        np.savez_compressed(a.out, features=np.concatenate([d["features"] for d in parts]),
                            log_ms=np.concatenate([d["log_ms"] for d in parts]),
                            patterns=np.concatenate([d["patterns"] for d in parts]), seed=int(parts[0]["seed"]),
                            plans=np.array(PLAN_NAMES))
        print(f"{nxt} entries -> {a.out}")
        return
    d = np.load(a.corpus)
    params, mean, scale, hist = train(d["features"], d["log_ms"], hidden=128, epochs=a.epochs, seed=a.seed,
                                      log_every=max(1, a.epochs // 10))
    save_weights(a.out, params, mean, scale, margin=a.margin, autotune=a.autotune)
    for ep, loss in hist:
        print(f"epoch {ep} loss {loss:.4f}")


if __name__ == "__main__":
    main()
