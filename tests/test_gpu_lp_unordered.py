"""phj_radix_lp's first run with unordered partition passes (phj_radix_bc's ranks), on the B200.

The first match among equal build keys depends on the order inside a build partition only when a probe
tuple has two or more matches. The join therefore first partitions as phj_radix_bc does and counts,
for every probe tuple, its matches; if one has two, it runs again with ordered passes (each build
partition in input order) and the result carries HJ_RES_ORDERED_PASSES. Every result here equals the
oracle's first-match join (src/algo/phj.c lp_join), whichever path ran."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
PIPELINES = {"segments": 0x20, "exact": 0x40}


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def unique_build(rng, n, kmax, rid_bits=32):
    keys = np.unique(rng.integers(1, kmax, 2 * n + 8, dtype=np.uint64))
    assert keys.shape[0] >= n
    R = np.empty((n, 2), dtype=np.uint64)
    R[:, 0] = rng.permutation(keys)[:n]
    R[:, 1] = rng.integers(0, 1 << rid_bits, n, dtype=np.uint64)
    return R


def probes(rng, R, n, miss_every=5, kmax=None):
    S = np.empty((n, 2), dtype=np.uint64)
    S[:, 0] = R[rng.integers(0, R.shape[0], n), 0]
    if kmax:
        S[::miss_every, 0] = rng.integers(1, kmax, S[::miss_every].shape[0], dtype=np.uint64)
    S[:, 1] = rng.integers(0, 1 << 32, n, dtype=np.uint64)
    return S


def run(hj, cuda, ctx, R, S, flags):
    return hj.join("phj_radix_lp", dev(cuda, R), dev(cuda, S), on_device=True, ctx=ctx, flags=flags)


@pytest.mark.parametrize("pipeline", list(PIPELINES))
def test_unique_build_keys_take_one_unordered_run(hj, oracle, cuda, pipeline):
    rng = np.random.default_rng(41)
    for nR, nS, kmax in [(200_000, 700_000, 1 << 22), (3_000, 9_000, 1 << 40), (1, 5, 4)]:
        R = unique_build(rng, nR, kmax)
        S = probes(rng, R, nS, kmax=kmax)
        with hj.Context(0) as ctx:
            r = run(hj, cuda, ctx, R, S, PIPELINES[pipeline])
        assert (r.matched_cnt, r.checksum) == oracle.join("phj_radix_lp", R, S), (nR, nS)
        assert not r.flags & hj.HJ_RES_ORDERED_PASSES


@pytest.mark.parametrize("pipeline", list(PIPELINES))
def test_duplicates_that_probes_hit_run_ordered(hj, oracle, cuda, pipeline):
    """Equal build keys spread over the relation (over many pass-1 CTAs and tiles): the unordered run
    finds a probe tuple with two matches, the join runs again ordered, and the next join of the same
    build relation on the context runs ordered at once."""
    rng = np.random.default_rng(42)
    R = unique_build(rng, 300_000, 1 << 22)
    R[150_000:150_600, 0] = R[:600, 0]  # 600 keys twice, far apart
    S = probes(rng, R, 800_000, kmax=1 << 22)
    want = oracle.join("phj_radix_lp", R, S)
    dR, dS = dev(cuda, R), dev(cuda, S)
    with hj.Context(0) as ctx:
        for i in range(2):
            r = hj.join("phj_radix_lp", dR, dS, on_device=True, ctx=ctx, flags=PIPELINES[pipeline])
            assert (r.matched_cnt, r.checksum) == want, i
            assert r.flags & hj.HJ_RES_ORDERED_PASSES, i


def test_duplicates_no_probe_hits_stay_unordered(hj, oracle, cuda):
    """Duplicate build keys that no probe tuple carries leave every first match unique."""
    rng = np.random.default_rng(43)
    R = unique_build(rng, 100_000, 1 << 21)
    dup_keys = R[:500, 0].copy()
    R[50_000:50_500, 0] = dup_keys
    S = probes(rng, R, 300_000)
    S = S[~np.isin(S[:, 0], dup_keys)]
    with hj.Context(0) as ctx:
        r = run(hj, cuda, ctx, R, S, 0)
    assert (r.matched_cnt, r.checksum) == oracle.join("phj_radix_lp", R, S)
    assert not r.flags & hj.HJ_RES_ORDERED_PASSES


@pytest.mark.parametrize("pipeline", list(PIPELINES))
def test_key_zero_never_matches(hj, oracle, cuda, pipeline):
    """Build key 0 is lp_join's empty slot: it never matches, in the unordered and the ordered passes,
    also when it occurs many times and probes carry it (no order dependence: none of them matches).
    Other keys of key 0's partition (radix bits 0, small high parts) must still match."""
    rng = np.random.default_rng(44)
    R = unique_build(rng, 120_000, 1 << 22)
    R[::97, 0] = 0
    # 2^22 + k * 2^14: radix bits 0 (key 0's partition), high parts 2^8 + k, no other build key
    R[5:25, 0] = np.uint64(1 << 22) + (np.arange(1, 21, dtype=np.uint64) << np.uint64(14))
    S = probes(rng, R, 400_000, kmax=1 << 22)
    S[::13, 0] = 0
    S[::17, 0] = R[5 + (np.arange(S[::17].shape[0]) % 20), 0]
    for rid_bits in (32, 48):  # compact words; 16-byte final partitions
        R2 = R.copy()
        R2[:, 1] = rng.integers(0, 1 << rid_bits, R.shape[0], dtype=np.uint64)
        want = oracle.join("phj_radix_lp", R2, S)
        for flags in (0, hj.HJ_F_ORDERED, hj.HJ_F_WORDS, hj.HJ_F_ORDERED | hj.HJ_F_WORDS):
            with hj.Context(0) as ctx:
                r = run(hj, cuda, ctx, R2, S, flags | PIPELINES[pipeline])
            assert (r.matched_cnt, r.checksum) == want, (rid_bits, flags)
            assert bool(r.flags & hj.HJ_RES_ORDERED_PASSES) == bool(flags & hj.HJ_F_ORDERED)
            assert bool(r.flags & hj.HJ_RES_COMPACT_PARTITIONS) == (rid_bits == 32)


def test_ordered_flag_and_wide_tuples(hj, oracle, cuda):
    rng = np.random.default_rng(45)
    R = unique_build(rng, 150_000, 1 << 22)
    R[70_000:70_300, 0] = R[:300, 0]
    S = probes(rng, R, 500_000, kmax=1 << 22)
    want = oracle.join("phj_radix_lp", R, S)
    for flags in (hj.HJ_F_ORDERED, hj.HJ_F_WIDE, hj.HJ_F_WORDS, hj.HJ_F_ORDERED | hj.HJ_F_WIDE):
        with hj.Context(0) as ctx:
            r = run(hj, cuda, ctx, R, S, flags)
        assert (r.matched_cnt, r.checksum) == want, flags
        assert r.flags & hj.HJ_RES_ORDERED_PASSES, flags


def test_hot_build_key_in_a_large_partition(hj, oracle, cuda):
    """A build key repeated 70,000 times lands in a partition joined through global memory (the
    key-aggregated table); probes that carry it have 70,000 matches, so the join runs ordered."""
    rng = np.random.default_rng(46)
    R = unique_build(rng, 200_000, 1 << 22)
    R[10_000:80_000, 0] = R[5, 0]
    S = probes(rng, R, 600_000, kmax=1 << 22)
    with hj.Context(0) as ctx:
        r = run(hj, cuda, ctx, R, S, 0)
    assert (r.matched_cnt, r.checksum) == oracle.join("phj_radix_lp", R, S)
    assert r.flags & hj.HJ_RES_ORDERED_PASSES
    assert r.large_partitions >= 1
    # the same build relation without probes on the hot key: one unordered run
    S2 = S[S[:, 0] != R[5, 0]]
    with hj.Context(0) as ctx:
        r = run(hj, cuda, ctx, R, S2, 0)
    assert (r.matched_cnt, r.checksum) == oracle.join("phj_radix_lp", R, S2)
    assert not r.flags & hj.HJ_RES_ORDERED_PASSES
