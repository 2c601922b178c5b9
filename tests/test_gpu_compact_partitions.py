"""Compact final partitions on the B200: when every build key shifted right by the radix bits is below
2^31 and every row id (build and probe) below 2^32, the last partition pass stores 8-byte words
(key >> bits) << 32 | row id and the joins read those (hj_result_t.flags has HJ_RES_COMPACT_PARTITIONS).
Results equal the oracle's on both sides of every limit, through both pipelines and the large-partition
path; joins with per-match output never use them."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
BITS = 14


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def rels(seed, nR=1 << 18, nS=1 << 20, kmax=1 << 24):
    rng = np.random.default_rng(seed)
    R = np.empty((nR, 2), dtype=np.uint64)
    R[:, 0] = rng.integers(1, kmax, nR, dtype=np.uint64)
    R[:, 1] = rng.integers(0, 1 << 32, nR, dtype=np.uint64)
    S = np.empty((nS, 2), dtype=np.uint64)
    S[:, 0] = R[rng.integers(0, nR, nS), 0]
    S[::7, 0] = rng.integers(1, kmax, S[::7].shape[0], dtype=np.uint64)
    S[:, 1] = rng.integers(0, 1 << 32, nS, dtype=np.uint64)
    return R, S


def run(hj, oracle, cuda, algo, R, S, flags=0, bits=BITS, passes=2):
    r = hj.join(algo, dev(cuda, R), dev(cuda, S), on_device=True, bits=bits, passes=passes, flags=flags)
    assert (r.matched_cnt, r.checksum) == oracle.join(algo, R, S), (algo, flags, bits, passes)
    return bool(r.flags & hj.HJ_RES_COMPACT_PARTITIONS)


@pytest.mark.parametrize("pipeline", ["exact", "segments"])
def test_flag_and_results_at_the_limits(hj, oracle, cuda, pipeline):
    flags = hj.HJ_F_SEGMENTS if pipeline == "segments" else hj.HJ_F_EXACT
    R, S = rels(1)
    assert run(hj, oracle, cuda, "phj_radix_bc", R, S, flags)
    # largest build key that fits: (2^31 - 1) << 14 | digits
    R2 = R.copy()
    R2[5, 0] = np.uint64(((1 << 31) - 1) << BITS | 77)
    S2 = S.copy()
    S2[3, 0] = R2[5, 0]
    assert run(hj, oracle, cuda, "phj_radix_bc", R2, S2, flags)
    # one build key past it: wide partitions
    R3 = R2.copy()
    R3[6, 0] = np.uint64((1 << 31) << BITS | 78)
    S3 = S2.copy()
    S3[4, 0] = R3[6, 0]
    assert not run(hj, oracle, cuda, "phj_radix_bc", R3, S3, flags)
    # a build row id of 2^32, or a probe row id of 2^32: wide
    R4 = R.copy()
    R4[9, 1] = np.uint64(1 << 32)
    assert not run(hj, oracle, cuda, "phj_radix_bc", R4, S, flags)
    S4 = S.copy()
    S4[9, 1] = np.uint64(1 << 32)
    assert not run(hj, oracle, cuda, "phj_radix_bc", R, S4, flags)
    # probe keys far beyond every build key (including all ones) stay compact and never match
    S5 = S.copy()
    S5[::5, 0] = np.uint64(2**64 - 1)
    S5[1::5, 0] = np.uint64((1 << 40) << BITS | 5)
    S5[2::5, 0] = np.uint64(((1 << 31) + 3) << BITS | 9)
    assert run(hj, oracle, cuda, "phj_radix_bc", R, S5, flags)


def test_other_names_and_geometries(hj, oracle, cuda):
    R, S = rels(2)
    R[::50, 0] = 0  # key 0: ignored by phj_radix_lp, a key like any other for the rest
    for algo in ("phj_radix_sc", "phj_radix_hr", "phj_asymm_radix_bc", "phj_radix_bw_reg_bc", "phj_radix_lp"):
        assert run(hj, oracle, cuda, algo, R, S)
    # one pass (8 bits) and two passes with an uneven split
    assert run(hj, oracle, cuda, "phj_radix_bc", R, S, bits=8, passes=1)
    assert run(hj, oracle, cuda, "phj_radix_bc", R, S, bits=11, passes=2)


def test_first_match_join_reads_compact_words(hj, oracle, cuda):
    """phj_radix_lp reads compact words: a build key 0 never matches (its words carry the high part
    0x80000000, which no build key has and no probe word gets: probe keys whose key >> bits is 2^31 or
    more are stored as 0xffffffff), and among duplicates the first build tuple in input order wins, in
    the compact, the 16-byte and the global-memory partition joins."""
    R, S = rels(4)
    R[::50, 0] = 0
    R[1::3, 0] = R[::3, 0][: R[1::3].shape[0]]          # duplicates: every key of R[::3] twice
    S[::11, 0] = 0                                       # probe key 0 finds nothing
    S[1::13, 0] = np.uint64((1 << 31) << BITS)           # partition 0, key >> bits = 2^31
    S[2::13, 0] = np.uint64(((1 << 31) + 5) << BITS | 3)
    for flags in (0, hj.HJ_F_EXACT):
        assert run(hj, oracle, cuda, "phj_radix_lp", R, S, flags)
    # partition 0 (the one key 0 lives in) with ~9000 and then ~16000 build tuples, key 0 and duplicates
    rng = np.random.default_rng(6)
    for n0 in (9000, 16000):
        base, _ = rels(7, nR=1 << 16, nS=1 << 17)
        p0 = np.empty((n0, 2), dtype=np.uint64)
        p0[:, 0] = rng.integers(0, 3000, n0, dtype=np.uint64) << np.uint64(BITS)
        p0[::40, 0] = 0
        p0[:, 1] = rng.integers(0, 1 << 32, n0, dtype=np.uint64)
        R2 = np.concatenate([p0[: n0 // 2], base, p0[n0 // 2:]])
        S2 = R2[rng.integers(0, R2.shape[0], 4 * R2.shape[0])].copy()
        S2[:, 1] = rng.integers(0, 1 << 32, S2.shape[0], dtype=np.uint64)
        S2[::17, 0] = np.uint64((1 << 31) << BITS)
        assert run(hj, oracle, cuda, "phj_radix_lp", R2, S2)


def test_mid_and_large_partitions_read_compact_words(hj, oracle, cuda):
    """Partitions above the compact shared-memory table (8192 build tuples) read compact words too:
    up to 10240 build tuples in the 16-byte shared-memory join, beyond that in the global-memory join,
    with duplicate keys and a hot key."""
    rng = np.random.default_rng(3)
    n_mid, n_big = 32 * 9000, 32 * 16000
    part = np.concatenate([rng.integers(0, 32, n_mid, dtype=np.uint64),      # ~9000 per partition
                           rng.integers(32, 64, n_big, dtype=np.uint64)])   # ~16000 per partition
    n = part.size
    R = np.empty((n, 2), dtype=np.uint64)
    R[:, 0] = (rng.integers(0, 5000, n, dtype=np.uint64) << np.uint64(BITS)) | part
    R[n_mid: n_mid + n_big // 8, 0] = np.uint64((7 << BITS) | 40)  # a hot key in a large partition
    R[:, 1] = rng.integers(0, 1 << 32, n, dtype=np.uint64)
    S = R[rng.integers(0, n, 2 * n)].copy()
    S[:, 1] = rng.integers(0, 1 << 32, S.shape[0], dtype=np.uint64)
    S[::9, 0] += np.uint64(1 << 30)
    for flags in (hj.HJ_F_EXACT, hj.HJ_F_SEGMENTS):
        assert run(hj, oracle, cuda, "phj_radix_bc", R, S, flags)


def test_headline_shape_uses_compact_partitions(hj, cuda):
    nR, nS = 1 << 22, 1 << 24
    R = cuda.empty((nR, 2), dtype=cuda.int64, device="cuda")
    S = cuda.empty((nS, 2), dtype=cuda.int64, device="cuda")
    hj.gen_fast_device(nR, nS, R.data_ptr(), S.data_ptr(), seed=3)
    cuda.cuda.synchronize()
    for flags in (0, hj.HJ_F_SEGMENTS, hj.HJ_F_EXACT):
        r = hj.join("phj_radix_bc", R, S, on_device=True, flags=flags)
        assert (r.matched_cnt, r.checksum) == hj.pkfk_closed_form(nR, nS)
        assert r.flags & hj.HJ_RES_COMPACT_PARTITIONS


def test_segment_mode_word_pass1_and_its_fallback(hj, oracle, cuda):
    """Segment mode stores pass 1 as 8-byte words when every build key >> b1 (7 of 14 bits here) is below
    2^31; otherwise pass 1 runs again with tuples on the device (counters reset), and the final partitions
    can still be compact (build keys >> 14 below 2^31). HJ_F_WIDE keeps tuples everywhere. Same results."""
    R, S = rels(5)
    # build keys in [2^38, 2^45): key >> 7 does not fit 31 bits, key >> 14 does
    R2 = R.copy()
    R2[:, 0] |= np.uint64(1 << 40)
    S2 = S.copy()
    S2[:, 0] |= np.uint64(1 << 40)
    for RR, SS in ((R, S), (R2, S2)):
        assert run(hj, oracle, cuda, "phj_radix_bc", RR, SS, hj.HJ_F_SEGMENTS)
        assert not run(hj, oracle, cuda, "phj_radix_bc", RR, SS, hj.HJ_F_SEGMENTS | hj.HJ_F_WIDE)
        assert not run(hj, oracle, cuda, "phj_radix_bc", RR, SS, hj.HJ_F_EXACT | hj.HJ_F_WIDE)
    # probe keys whose key >> 7 does not fit: kept as non-matching words, their digits intact
    S3 = S.copy()
    S3[::3, 0] = np.uint64(((1 << 45) + 12345) << 7) | (S3[::3, 0] & np.uint64(0x3FFF))
    assert run(hj, oracle, cuda, "phj_radix_bc", R, S3, hj.HJ_F_SEGMENTS)
    # the stall hook still reports the expired wait with word passes
    with pytest.raises(hj.JoinError) as e:
        hj.join("phj_radix_bc", dev(cuda, R), dev(cuda, S), on_device=True, flags=hj.HJ_F_SEGMENTS | hj.HJ_F_TEST_STALL)
    assert e.value.status == hj.HJ_E_TIMEOUT
    assert run(hj, oracle, cuda, "phj_radix_bc", R, S, hj.HJ_F_SEGMENTS)  # the context recovers


@pytest.mark.parametrize("algo", ["phj_radix_bc", "phj_radix_lp"])
def test_exact_pipeline_word_pass1(hj, oracle, cuda, algo):
    """The exact-offset pipeline stores pass 1 as 8-byte words too when the histogram pass's ORs allow
    them (by default only for large units; HJ_F_WORDS asks for it here); pass 2 then reads its units at
    word offsets, odd ones included (a tile's copy starts one word early). Build keys too wide for pass-1 words keep tuples in pass 1 (the final partitions can still be
    compact); HJ_F_WIDE keeps tuples everywhere. Results equal the oracle's, with duplicates and key 0."""
    R, S = rels(9)
    R[::37, 0] = 0
    R[1::5, 0] = R[::5, 0][: R[1::5].shape[0]]
    R2 = R.copy()
    S2 = S.copy()
    R2[:, 0] |= np.uint64(1 << 40)  # key >> 7 does not fit 31 bits, key >> 14 does
    S2[:, 0] |= np.uint64(1 << 40)
    for RR, SS, words in ((R, S, True), (R2, S2, False)):
        want = oracle.join(algo, RR, SS)
        for bits, b1 in ((14, 7), (12, 5), (9, 4)):
            r = hj.join(algo, dev(cuda, RR), dev(cuda, SS), on_device=True, bits=bits, passes=2,
                        bits_pass1=b1, flags=hj.HJ_F_EXACT | hj.HJ_F_WORDS)
            assert (r.matched_cnt, r.checksum) == want, (algo, bits, b1, words)
            assert bool(r.flags & hj.HJ_RES_WORD_PASS1) == words, (bits, b1)
        r = hj.join(algo, dev(cuda, RR), dev(cuda, SS), on_device=True, flags=hj.HJ_F_EXACT | hj.HJ_F_WIDE)
        assert (r.matched_cnt, r.checksum) == want
        assert not r.flags & hj.HJ_RES_WORD_PASS1
        # by default these small units keep tuples in pass 1
        r = hj.join(algo, dev(cuda, RR), dev(cuda, SS), on_device=True, flags=hj.HJ_F_EXACT)
        assert (r.matched_cnt, r.checksum) == want
        assert not r.flags & hj.HJ_RES_WORD_PASS1
