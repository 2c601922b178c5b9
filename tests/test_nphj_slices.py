"""CPU restatement of the index arithmetic of the non-partitioned join's sliced build (hj_nphj.cu:
nphj_widths, nphj_slice_colscan, nphj_slice_plan, nphj_slice_scatter, nphj_slice_build and the probe's
slice wrap), run before the kernels ever touch a GPU: every staging write lands inside [0, |R|) exactly
once, each slice holds only its own keys, no slice overflows its slots, and probing inside slices gives
the oracle's result, for every-match joins (staged key and row id) and first-match joins (staged key and
input position, smallest position kept per key, then its row id)."""
import numpy as np
import pytest

M64 = (1 << 64) - 1
SLICE_LOG = 13
SLICE = 1 << SLICE_LOG
MAX_FILL = SLICE // 8 * 7


def table_hash(key, cap):
    h = (key * 0x9E3779B97F4A7C15) & M64
    h ^= h >> 29
    h = (h * 0xBF58476D1CE4E5B9) & M64
    h ^= h >> 32
    return (h * cap) >> 64


def sliced_join(R, S, hist_blocks, lp=False):
    nR = R.shape[0]
    cap = int(nR / 0.5) + 2
    ccap = (cap + SLICE - 1) // SLICE * SLICE
    ns = ccap // SLICE
    keys = [int(k) for k in R[:, 0]]
    rids = [int(r) for r in R[:, 1]]
    sl = [table_hash(k, ccap) >> SLICE_LOG for k in keys]
    assert all(0 <= x < ns for x in sl)
    # nphj_widths: block b counts its contiguous range [b*per, min(nR, (b+1)*per))
    per = (nR + hist_blocks - 1) // hist_blocks
    hist = np.zeros((hist_blocks, ns), dtype=np.int64)
    for b in range(hist_blocks):
        lo, hi = min(nR, b * per), min(nR, b * per + per)
        for i in range(lo, hi):
            hist[b, sl[i]] += 1
    # nphj_slice_colscan: exclusive scan down each column; nphj_slice_plan: slice starts
    off = np.cumsum(hist, axis=0) - hist
    total = hist.sum(axis=0)
    start = np.concatenate([[0], np.cumsum(total)])
    assert start[-1] == nR and total.max() <= MAX_FILL
    # nphj_slice_scatter: block b writes its tuples of slice s from start[s] + off[b][s] on
    stage = [None] * nR
    for b in range(hist_blocks):
        pos = start[:-1] + off[b]
        lo, hi = min(nR, b * per), min(nR, b * per + per)
        for i in range(lo, hi):
            p = int(pos[sl[i]])
            pos[sl[i]] += 1
            assert 0 <= p < nR and stage[p] is None
            stage[p] = (keys[i] << 32) | (i if lp else rids[i])
    assert all(v is not None for v in stage)
    # nphj_slice_build: per slice, linear probing inside the slice
    table = [None] * ccap
    for s in range(ns):
        for v in stage[start[s]:start[s + 1]]:
            k = v >> 32
            assert table_hash(k, ccap) >> SLICE_LOG == s
            h = table_hash(k, ccap) & (SLICE - 1)
            for _ in range(SLICE):
                cur = table[s * SLICE + h]
                if cur is None:
                    table[s * SLICE + h] = v
                    break
                if lp and cur >> 32 == k:  # first match: the smallest position per key
                    table[s * SLICE + h] = min(cur, v)
                    break
                h = (h + 1) & (SLICE - 1)
            else:
                raise AssertionError("slice overflow")
    if lp:  # positions -> row ids
        table = [None if e is None else (e & ~0xFFFFFFFF) | rids[e & 0xFFFFFFFF] for e in table]
    # probe with the slice wrap (every match: nphj_sc)
    cnt = csum = 0
    for k, r in zip(S[:, 0], S[:, 1]):
        k, r = int(k), int(r)
        if k >= 0xFFFFFFFF:
            continue
        h = table_hash(k, ccap)
        for _ in range(SLICE):
            e = table[h]
            if e is None:
                break
            if e >> 32 == k:
                cnt += 1
                csum = (csum + (e & 0xFFFFFFFF) + r) & M64
                if lp:
                    break
            h = (h & ~(SLICE - 1)) | ((h + 1) & (SLICE - 1))
    return cnt, csum


@pytest.mark.parametrize("lp", [False, True])
@pytest.mark.parametrize("nR,nS,hist_blocks,dups", [(20_000, 50_000, 7, False), (30_001, 40_000, 296, True),
                                                    (8_192, 20_000, 1, True)])
def test_sliced_build_index_arithmetic(oracle, nR, nS, hist_blocks, dups, lp):
    rng = np.random.default_rng(nR)
    R = np.empty((nR, 2), dtype=np.uint64)
    R[:, 0] = rng.integers(1, nR // 3 if dups else 1 << 31, nR, dtype=np.uint64)
    R[:, 1] = rng.integers(0, 1 << 32, nR, dtype=np.uint64)
    S = np.empty((nS, 2), dtype=np.uint64)
    S[:, 0] = R[rng.integers(0, nR, nS), 0]
    S[::9, 0] = rng.integers(1, 1 << 33, S[::9].shape[0], dtype=np.uint64)
    S[:, 1] = rng.integers(0, 1 << 40, nS, dtype=np.uint64)
    assert sliced_join(R, S, hist_blocks, lp) == oracle.join("nphj_lp" if lp else "nphj_sc", R, S)
