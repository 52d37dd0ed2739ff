"""Block-sparse tensors and their block-task lists.

A block-sparse tensor splits every index into segments; a block is one
combination of segments, stored densely in TAL-SH's "dlf" layout.  The task
list of a contraction pairs every present left block with every present right
block that agrees on the contracted segments, which is the work ExaTENSOR's
hierarchical layer hands to TAL-SH one block at a time
(INTERVIRT/tavp_worker.F90:9420, via INTRAVIRT/tensor_recursive.F90's block
decomposition).  The list feeds :class:`exatensor_b200.BlockSparsePlan`.

Device memory comes from torch (one buffer per tensor); nothing here computes.
"""
from __future__ import annotations

import itertools
import re

import numpy as np


def _labels(pattern: str):
    groups = re.findall(r"\(([^)]*)\)", pattern)
    if len(groups) != 3:
        raise ValueError("a contraction pattern D(...)+=L(...)*R(...) is required")
    return [[x.strip().rstrip("+") for x in g.split(",")] if g.strip() else [] for g in groups]


class BlockSparseTensor:
    """Blocks of a tensor whose index k is split into ``segments[k]`` (extents).

    ``blocks`` maps a block key (tuple of segment numbers) to
    (element offset, extents) inside one device buffer ``data``."""

    def __init__(self, segments, keys, elem_bytes, device="cuda"):
        import torch
        self.segments = [list(s) for s in segments]
        self.elem_bytes = elem_bytes
        self.blocks = {}
        off = 0
        for key in sorted(set(keys)):
            dims = [self.segments[k][s] for k, s in enumerate(key)]
            vol = int(np.prod(dims))
            self.blocks[key] = (off, dims)
            off += (vol + 31) // 32 * 32  # keep every block 256-byte aligned
        self.volume = off
        self.data = torch.zeros(max(1, off) * elem_bytes, dtype=torch.uint8, device=device)

    def ptr(self, key) -> int:
        return self.data.data_ptr() + self.blocks[key][0] * self.elem_bytes

    def dims(self, key):
        return self.blocks[key][1]


def random_segments(rank, nseg, lo, hi, rng):
    return [[int(x) for x in rng.integers(lo, hi + 1, size=nseg)] for _ in range(rank)]


def random_keys(segments, presence, rng):
    keys = list(itertools.product(*[range(len(s)) for s in segments]))
    keep = rng.random(len(keys)) < presence
    return [k for k, m in zip(keys, keep) if m]


def contraction_tasks(pattern, L: BlockSparseTensor, R: BlockSparseTensor, d_segments=None, elem_bytes=None,
                      device="cuda"):
    """Output tensor (blocks that receive at least one product) and the task
    list ``[(d_ptr, d_dims, l_ptr, l_dims, r_ptr, r_dims), ...]``."""
    dl, ll, rl = _labels(pattern)
    contracted = [x for x in ll if x in rl]
    lpos = {x: i for i, x in enumerate(ll)}
    rpos = {x: i for i, x in enumerate(rl)}
    seg_of = {}
    for x in ll:
        seg_of[x] = L.segments[lpos[x]]
    for x in rl:
        seg_of.setdefault(x, R.segments[rpos[x]])
    # right blocks by their contracted segments
    rby = {}
    for rk in R.blocks:
        rby.setdefault(tuple(rk[rpos[x]] for x in contracted), []).append(rk)
    pairs = []
    for lk in L.blocks:
        c = tuple(lk[lpos[x]] for x in contracted)
        for rk in rby.get(c, []):
            dkey = tuple(lk[lpos[x]] if x in lpos else rk[rpos[x]] for x in dl)
            pairs.append((dkey, lk, rk))
    D = BlockSparseTensor(d_segments or [seg_of[x] for x in dl], [p[0] for p in pairs],
                          elem_bytes or L.elem_bytes, device)
    tasks = [(D.ptr(dk), D.dims(dk), L.ptr(lk), L.dims(lk), R.ptr(rk), R.dims(rk)) for dk, lk, rk in pairs]
    return D, tasks, pairs
