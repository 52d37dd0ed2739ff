"""The block-task producer (tb_bsc_tasks_from_blocks, host code) against a
plain restatement of the matching that ExaTENSOR's TensContractionSplitFunc
does (INTRAVIRT/tensor_recursive.F90:9202-9784): every (L block, R block)
pair whose contracted segments agree yields one task on the D block named by
their uncontracted segments, if D holds it.  Block bodies are stand-in
addresses: nothing is dereferenced."""
import itertools
import re

import numpy as np
import pytest

import exatensor_b200 as XB


def labels(pattern):
    g = re.findall(r"\(([^)]*)\)", pattern)
    return [[x.strip() for x in s.split(",")] if s.strip() else [] for s in g]


def expected_tasks(pattern, d, l, r):
    dl, ll, rl = labels(pattern)
    lpos = {x: i for i, x in enumerate(ll)}
    rpos = {x: i for i, x in enumerate(rl)}
    contracted = [x for x in rl if x in lpos]
    dkeys = {tuple(k): i for i, k in enumerate(d[1])}
    out = []
    for i, lk in enumerate(l[1]):
        for j, rk in enumerate(r[1]):
            if any(lk[lpos[x]] != rk[rpos[x]] for x in contracted):
                continue
            dk = tuple(lk[lpos[x]] if x in lpos else rk[rpos[x]] for x in dl)
            if dk not in dkeys:
                continue
            di = dkeys[dk]
            out.append((d[2][di], [d[0][p][dk[p]] for p in range(len(dl))], l[2][i],
                        [l[0][a][lk[a]] for a in range(len(ll))], r[2][j],
                        [r[0][b][rk[b]] for b in range(len(rl))]))
    return out


def block_tensor(segments, presence, rng, base):
    keys = [k for k in itertools.product(*[range(len(s)) for s in segments]) if rng.random() < presence]
    return segments, keys, [base + 4096 * i for i in range(len(keys))]


@pytest.mark.parametrize("pattern", ["D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)", "D(a,i,b,j)+=L(a,k,c,i)*R(c,b,k,j)",
                                     "D(i,j)+=L(k,i)*R(k,j)", "D(a,b,c)+=L(c,k,a)*R(k,b)"])
@pytest.mark.parametrize("seed", [0, 1])
def test_tasks_match_the_restated_matching(pattern, seed):
    rng = np.random.default_rng(seed)
    dl, ll, rl = labels(pattern)
    seg = {x: [int(v) for v in rng.integers(2, 9, size=int(rng.integers(2, 4)))] for x in set(dl + ll + rl)}
    L = block_tensor([seg[x] for x in ll], 0.6, rng, 1 << 32)
    R = block_tensor([seg[x] for x in rl], 0.6, rng, 2 << 32)
    D = block_tensor([seg[x] for x in dl], 0.8, rng, 3 << 32)
    got = XB.bsc_tasks_from_blocks(pattern, D, L, R)
    exp = expected_tasks(pattern, D, L, R)
    assert len(exp) > 0
    assert got == exp


def test_pairs_without_an_output_block_give_no_task():
    pattern = "D(i,j)+=L(k,i)*R(k,j)"
    s = [[4, 4], [3, 5]]
    L = (s, [(0, 0), (1, 1)], [10, 11])
    R = ([[4, 4], [2]], [(0, 0), (1, 0)], [20, 21])
    D = ([[3, 5], [2]], [(0, 0)], [30])
    got = XB.bsc_tasks_from_blocks(pattern, D, L, R)
    assert got == [(30, [3, 2], 10, [4, 3], 20, [4, 2])]


def test_bad_metadata_is_rejected():
    pattern = "D(i,j)+=L(k,i)*R(k,j)"
    L = ([[4, 4], [3, 5]], [(0, 0)], [10])
    R = ([[4, 5], [2]], [(0, 0)], [20])          # k segmented unlike L's k
    D = ([[3, 5], [2]], [(0, 0)], [30])
    with pytest.raises(XB.TBError):
        XB.bsc_tasks_from_blocks(pattern, D, L, R)
    R_ok = ([[4, 4], [2]], [(0, 0)], [20])
    with pytest.raises(XB.TBError):                # segment number out of range
        XB.bsc_tasks_from_blocks(pattern, D, ([[4, 4], [3, 5]], [(0, 2)], [10]), R_ok)
    with pytest.raises(XB.TBError):                # repeated D key
        XB.bsc_tasks_from_blocks(pattern, ([[3, 5], [2]], [(0, 0), (0, 0)], [30, 31]), L, R_ok)
    with pytest.raises(XB.TBError):                # ranks do not match the pattern
        XB.bsc_tasks_from_blocks(pattern, ([[3, 5]], [(0,)], [30]), L, R_ok)


def test_too_small_a_task_array_reports_the_count():
    import ctypes as C
    pattern = "D(i,j)+=L(k,i)*R(k,j)"
    L = ([[4, 4], [3, 5]], [(0, 0), (0, 1), (1, 0)], [10, 11, 12])
    R = ([[4, 4], [2]], [(0, 0), (1, 0)], [20, 21])
    D = ([[3, 5], [2]], [(0, 0), (1, 0)], [30, 31])
    bd, kd = XB._block_list(*D)
    bl, kl = XB._block_list(*L)
    br, kr = XB._block_list(*R)
    arr = (XB.BlockTask * 1)()
    n = C.c_int()
    code = XB.lib().tb_bsc_tasks_from_blocks(pattern.encode(), C.byref(bd), C.byref(bl), C.byref(br), 1, arr,
                                             C.byref(n))
    assert code == 7 and n.value == 3  # TB_ERR_LIMIT, with the count needed
