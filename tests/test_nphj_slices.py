"""CPU restatement of the index arithmetic of the non-partitioned join's sliced build (hj_nphj.cu:
nphj_slice_scatter, nphj_slice_build and the probe's slice wrap), run before the kernels ever touch a
GPU: each block counts its contiguous range of R per slice, claims space in every slice's staging area
(kSliceMaxFill words) in whatever order the blocks reach the atomic, and writes at its claim plus a rank;
every staging write lands inside its slice's area exactly once, each slice holds only its own keys, and
probing inside slices gives the oracle's result whatever the claim order, for every-match joins (staged
key and row id) and first-match joins (staged key and input position, smallest position kept per key,
then its row id)."""
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


def default_load(nR):
    """nphj_default_load: the table load factor a table_load of 0 selects."""
    return 0.4 if nR <= 5_000_000 else 0.5


def table_cap(nR, load):
    """nphj_cap: 16-byte table slots for nR build tuples."""
    return int(nR / load) + 2


def compact_used(nR, load):
    """nphj_enqueue's compact_ok for a join without per-match output or the key-0 rule: the 16-byte table
    would exceed 64 MB."""
    return table_cap(nR, load) * 16 > (64 << 20)


def staging_fits(nR, load=0.5):
    """The host's test (nphj_enqueue): the compact table, the staging areas and the fill counters fit in the
    16-byte table's bytes. True for every table the sliced build is used for (above 64 MB the rounding of
    the capacity to whole slices is below 0.2%); small or badly rounded tables build without slices."""
    a256 = lambda x: (x + 255) // 256 * 256
    cap = table_cap(nR, load)
    ccap = (cap + SLICE - 1) // SLICE * SLICE
    ns = ccap // SLICE
    return a256(ccap * 8) + a256(ns * MAX_FILL * 8) + ns * 4 <= cap * 16


def sliced_join(R, S, hist_blocks, lp=False, claim_seed=0, load=0.5):
    nR = R.shape[0]
    cap = table_cap(nR, load)
    ccap = (cap + SLICE - 1) // SLICE * SLICE
    ns = ccap // SLICE
    keys = [int(k) for k in R[:, 0]]
    rids = [int(r) for r in R[:, 1]]
    sl = [table_hash(k, ccap) >> SLICE_LOG for k in keys]
    assert all(0 <= x < ns for x in sl)
    assert staging_fits(nR, load)  # otherwise the host builds without slices
    # pass 1 of nphj_slice_scatter: block b counts its contiguous range [b*per, min(nR, (b+1)*per))
    per = (nR + hist_blocks - 1) // hist_blocks
    hist = np.zeros((hist_blocks, ns), dtype=np.int64)
    for b in range(hist_blocks):
        lo, hi = min(nR, b * per), min(nR, b * per + per)
        for i in range(lo, hi):
            hist[b, sl[i]] += 1
    # claims: one atomic per (block, slice), blocks in an arbitrary order
    fill = np.zeros(ns, dtype=np.int64)
    base = np.zeros((hist_blocks, ns), dtype=np.int64)
    for b in np.random.default_rng(claim_seed).permutation(hist_blocks):
        base[b] = fill
        fill += hist[b]
    assert fill.sum() == nR and fill.max() <= MAX_FILL  # no overflow: the build is sliced
    # pass 2: block b writes its tuples of slice s at s * MAX_FILL + its claim + a rank
    stage = [None] * (ns * MAX_FILL)
    for b in range(hist_blocks):
        pos = base[b].copy()
        lo, hi = min(nR, b * per), min(nR, b * per + per)
        for i in range(lo, hi):
            s = sl[i]
            p = int(pos[s])
            pos[s] += 1
            assert 0 <= p < MAX_FILL and stage[s * MAX_FILL + p] is None
            stage[s * MAX_FILL + p] = (keys[i] << 32) | (i if lp else rids[i])
    assert sum(v is not None for v in stage) == nR
    # nphj_slice_build: per slice, linear probing inside the slice
    table = [None] * ccap
    for s in range(ns):
        for v in stage[s * MAX_FILL:s * MAX_FILL + int(fill[s])]:
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
@pytest.mark.parametrize("nR,nS,hist_blocks,dups", [(20_478, 50_000, 7, False), (28_670, 40_000, 296, True),
                                                    (8_190, 20_000, 1, True)])
def test_sliced_build_index_arithmetic(oracle, nR, nS, hist_blocks, dups, lp):
    rng = np.random.default_rng(nR)
    R = np.empty((nR, 2), dtype=np.uint64)
    R[:, 0] = rng.integers(1, nR // 3 if dups else 1 << 31, nR, dtype=np.uint64)
    R[:, 1] = rng.integers(0, 1 << 32, nR, dtype=np.uint64)
    S = np.empty((nS, 2), dtype=np.uint64)
    S[:, 0] = R[rng.integers(0, nR, nS), 0]
    S[::9, 0] = rng.integers(1, 1 << 33, S[::9].shape[0], dtype=np.uint64)
    S[:, 1] = rng.integers(0, 1 << 40, nS, dtype=np.uint64)
    want = oracle.join("nphj_lp" if lp else "nphj_sc", R, S)
    for seed in (0, 1):  # two claim orders
        assert sliced_join(R, S, hist_blocks, lp, seed) == want


def test_staging_fits_every_table_the_sliced_build_is_used_for():
    # compact tables are used above 64 MB of 16-byte slots (nR > 2^21 at load 0.5)
    for nR in (1 << 21, (1 << 21) + 1, 3_000_001, 1 << 22, 10**7 + 7, 1 << 26):
        assert staging_fits(nR), nR
    assert not staging_fits(30_001)  # a small, badly rounded table: the host builds without slices
    # the default load factors (0.4 up to 5 M build tuples, 0.5 above) and a few others, over sizes
    # from 2^20 to 2^30: wherever the compact table is used, the staging fits
    for load in (None, 0.3, 0.4, 0.5, 0.7):
        for nR in np.unique(np.geomspace(1 << 20, 1 << 30, 400).astype(np.int64)).tolist() + [5_000_000, 5_000_001]:
            ld = default_load(nR) if load is None else load
            if compact_used(nR, ld):
                assert staging_fits(nR, ld), (nR, ld)


def test_expected_slice_fill_at_the_default_loads():
    """A slice holds kSliceSlots * load build tuples on average; its staging area holds 7/8 of the slice.
    With uniform hashing over many slices the fill is about Poisson, so at load 0.5 the area's bound lies
    48 standard deviations above the mean and at 0.4 68: only repeated keys overflow a slice (then the
    global-CAS build runs)."""
    for load, sigmas in ((0.4, 68), (0.5, 48)):
        mean = SLICE * load
        assert round((MAX_FILL - mean) / mean ** 0.5) == sigmas, load


def test_sliced_build_at_load_0_4(oracle):
    """The index arithmetic at the small-table default load, on a table large enough for its staging."""
    rng = np.random.default_rng(5)
    nR, nS = 60_000, 90_000
    assert staging_fits(nR, 0.4)
    R = np.empty((nR, 2), dtype=np.uint64)
    R[:, 0] = rng.integers(1, 1 << 31, nR, dtype=np.uint64)
    R[:, 1] = rng.integers(0, 1 << 32, nR, dtype=np.uint64)
    S = np.empty((nS, 2), dtype=np.uint64)
    S[:, 0] = R[rng.integers(0, nR, nS), 0]
    S[:, 1] = rng.integers(0, 1 << 40, nS, dtype=np.uint64)
    for lp in (False, True):
        assert sliced_join(R, S, 37, lp, 3, load=0.4) == oracle.join("nphj_lp" if lp else "nphj_sc", R, S)
