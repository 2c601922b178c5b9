"""GPU parity of segment mode: the radix joins partition in pass 1 into chains of fixed-size segments
and count the histograms on the way (no histogram pass). Forced at
small sizes with HJ_F_SEGMENTS, its results must equal the oracle's and the exact-offset pipeline's
(HJ_F_EXACT) bit for bit, on uniform, skewed, duplicate-heavy and ragged inputs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ALL_MATCH = ["phj_radix_bc", "phj_radix_sc", "phj_radix_hr", "phj_radix_hro"]


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def random_rel(rng, n, lo, hi):
    a = np.empty((n, 2), dtype=np.uint64)
    a[:, 0] = rng.integers(lo, hi, n, dtype=np.uint64, endpoint=True)
    a[:, 1] = rng.integers(0, 2**64 - 1, n, dtype=np.uint64, endpoint=True)
    return a


def both(hj, cuda, algo, R, S, **kw):
    dR, dS = dev(cuda, R), dev(cuda, S)
    seg = hj.join(algo, dR, dS, on_device=True, flags=hj.HJ_F_SEGMENTS | hj.HJ_F_PHASE_TIMES, **kw)
    exact = hj.join(algo, dR, dS, on_device=True, flags=hj.HJ_F_EXACT | hj.HJ_F_PHASE_TIMES, **kw)
    return seg, exact


@pytest.mark.parametrize("algo", ALL_MATCH)
def test_segment_mode_matches_oracle(hj, oracle, cuda, algo):
    rng = np.random.default_rng(11)
    cases = [
        (random_rel(rng, 50_000, 1, 200_000), random_rel(rng, 120_000, 1, 200_000)),
        (random_rel(rng, 1, 1, 10), random_rel(rng, 1, 1, 10)),
        (random_rel(rng, 2047, 1, 5000), random_rel(rng, 2049, 1, 5000)),        # ragged last tiles
        (random_rel(rng, 30_000, 1, 40), random_rel(rng, 70_000, 1, 60)),        # one digit per tile run
        (random_rel(rng, 20_000, 0, 5), random_rel(rng, 9_000, 0, 6)),           # key 0, few keys
        (random_rel(rng, 100_000, 1, 2**62), random_rel(rng, 5, 1, 2**62)),      # almost only R
    ]
    for R, S in cases:
        want = oracle.join(algo, R, S)
        seg, exact = both(hj, cuda, algo, R, S)
        assert (seg.matched_cnt, seg.checksum) == want, (algo, len(R), len(S))
        assert (exact.matched_cnt, exact.checksum) == want
        assert seg.phase[0] == 0.0 and seg.phase[2] > 0.0  # no histogram pass; pass 1 timed
        assert exact.phase[0] > 0.0


@pytest.mark.parametrize("bits,b1", [(2, 1), (9, 4), (12, 8), (14, 7), (14, 6), (13, 5)])
def test_segment_mode_geometries(hj, oracle, cuda, bits, b1):
    rng = np.random.default_rng(bits * 31 + b1)
    R = random_rel(rng, 80_000, 1, 300_000)
    S = random_rel(rng, 200_000, 1, 300_000)
    want = oracle.join("phj_radix_bc", R, S)
    seg, exact = both(hj, cuda, "phj_radix_bc", R, S, bits=bits, passes=2, bits_pass1=b1)
    assert (seg.matched_cnt, seg.checksum) == want
    assert (exact.matched_cnt, exact.checksum) == want


def test_segment_mode_skew(hj, oracle, cuda):
    # Zipf-like probe keys over a PK build side, and a build side where one key holds a third of R:
    # single digits take whole tiles and chains grow long.
    rng = np.random.default_rng(3)
    nR = 1 << 16
    R = np.empty((nR, 2), dtype=np.uint64)
    R[:, 0] = rng.permutation(np.arange(1, nR + 1, dtype=np.uint64))
    R[:, 1] = rng.integers(0, 2**63, nR, dtype=np.uint64)
    z = np.minimum(rng.zipf(1.3, 600_000), nR).astype(np.uint64)
    S = np.stack([z, rng.integers(0, 2**63, z.size, dtype=np.uint64)], axis=1)
    R2 = R.copy()
    R2[: nR // 3, 0] = 4242
    for r in (R, R2):
        want = oracle.join("phj_radix_bc", r, S)
        seg, _ = both(hj, cuda, "phj_radix_bc", r, S)
        assert (seg.matched_cnt, seg.checksum) == want


def test_segment_mode_hot_bin(hj, cuda):
    # Every key has the same low 14 bits: one partition gets everything, each pass-1 CTA counts far
    # more than 32768 tuples into one 16-bit counter (which must spill into its row), and the join
    # takes the large-partition path. Unique build keys, probe keys drawn from them.
    rng = np.random.default_rng(21)
    nR, nS = 1 << 22, 1 << 24
    R = np.empty((nR, 2), dtype=np.uint64)
    R[:, 0] = (rng.permutation(nR).astype(np.uint64) + np.uint64(1)) << np.uint64(14) | np.uint64(7)
    R[:, 1] = rng.integers(0, 2**63, nR, dtype=np.uint64)
    pick = rng.integers(0, nR, nS)
    S = np.stack([R[pick, 0], rng.integers(0, 2**63, nS, dtype=np.uint64)], axis=1)
    with np.errstate(over="ignore"):
        want = (nS, int((R[pick, 1].sum(dtype=np.uint64) + S[:, 1].sum(dtype=np.uint64))))
    seg, exact = both(hj, cuda, "phj_radix_bc", R, S)
    assert (seg.matched_cnt, seg.checksum) == want
    assert (exact.matched_cnt, exact.checksum) == want
    assert seg.large_partitions == 1


def narrow(a):
    """Row ids below 2^32: with small keys the 8-byte word layout applies."""
    a = a.copy()
    a[:, 1] &= np.uint64(0xFFFFFFFF)
    return a


def test_segment_mode_first_match(hj, oracle, cuda):
    """phj_radix_lp in segment mode: each pass-1 CTA takes a contiguous range of the build relation, in
    order, and ranks its tiles stably, and pass 2 writes each digit's chains in CTA order, so every
    final build partition keeps input order and the first match is the reference's. Duplicates spread
    over the whole build relation (over many pass-1 CTAs), key 0, ragged tiles; 16-byte tuples, 8-byte
    words in pass 1 and the final partitions, and build keys too wide for pass-1 words (pass 1 runs
    again with tuples)."""
    rng = np.random.default_rng(8)
    cases = [
        (random_rel(rng, 40_000, 1, 10_000), random_rel(rng, 90_000, 1, 12_000), False),
        (narrow(random_rel(rng, 300_000, 0, 3_000)), narrow(random_rel(rng, 200_000, 0, 3_500)), True),
        (narrow(random_rel(rng, 2047, 0, 50)), narrow(random_rel(rng, 4099, 0, 60)), True),
        (narrow(random_rel(rng, 1, 0, 0)), narrow(random_rel(rng, 3, 0, 0)), True),
        (random_rel(rng, 250_000, 0, 2_000), random_rel(rng, 100_000, 0, 2_200), False),
    ]
    wide = narrow(random_rel(rng, 100_000, 0, 4_000))
    wide[:, 0] = (wide[:, 0] << np.uint64(40)) | (wide[:, 0] & np.uint64(0x3FFF))  # key >> 7 beyond 2^31
    wide[::97, 0] = 0
    wide_s = wide[rng.integers(0, wide.shape[0], 150_000)].copy()
    wide_s[:, 1] = rng.integers(0, 1 << 32, wide_s.shape[0], dtype=np.uint64)
    cases.append((wide, wide_s, False))
    for R, S, words in cases:
        want = oracle.join("phj_radix_lp", R, S)
        seg, exact = both(hj, cuda, "phj_radix_lp", R, S)
        assert (seg.matched_cnt, seg.checksum) == want, (len(R), len(S))
        assert (exact.matched_cnt, exact.checksum) == want
        assert seg.phase[0] == 0.0 and exact.phase[0] > 0.0  # no histogram pass in segment mode
        assert bool(seg.flags & hj.HJ_RES_WORD_PASS1) == words


def test_segment_mode_first_match_pairs(hj, oracle, cuda):
    """The materialising first-match join in segment mode writes the reference's pairs."""
    rng = np.random.default_rng(21)
    R = np.empty((60_000, 2), dtype=np.uint64)
    R[:, 0] = rng.integers(0, 5_000, R.shape[0], dtype=np.uint64)
    R[:, 1] = np.arange(1, R.shape[0] + 1, dtype=np.uint64)  # row ids: 1-based positions (retrieve)
    S = np.empty((90_000, 2), dtype=np.uint64)
    S[:, 0] = rng.integers(0, 5_500, S.shape[0], dtype=np.uint64)
    S[:, 1] = np.arange(1, S.shape[0] + 1, dtype=np.uint64)
    want = oracle.join_pairs("ptr_phj_radix_lp", R, S)
    out = cuda.zeros((want.shape[0] + 10, 2), dtype=cuda.int64, device="cuda")
    r = hj.join_mat("ptr_phj_radix_lp", dev(cuda, R), dev(cuda, S), pairs=out, on_device=True,
                    flags=hj.HJ_F_SEGMENTS)
    assert r.matched_cnt == want.shape[0]
    got = out[: r.matched_cnt].cpu().numpy().view(np.uint64)
    got = got[np.lexsort((got[:, 1], got[:, 0]))]
    assert np.array_equal(got, want)


def test_segment_mode_first_match_large_partitions(hj, oracle, cuda):
    """First-match joins in segment mode with build partitions above the shared-memory tables (the
    global-memory join keeps the lowest position among equal keys), with key 0 among them."""
    rng = np.random.default_rng(22)
    n = 64 * 12_000
    R = np.empty((n, 2), dtype=np.uint64)
    R[:, 0] = (rng.integers(0, 6_000, n, dtype=np.uint64) << np.uint64(14)) | rng.integers(0, 64, n, dtype=np.uint64)
    R[::50, 0] = 0
    R[:, 1] = rng.integers(0, 1 << 32, n, dtype=np.uint64)
    S = R[rng.integers(0, n, 2 * n)].copy()
    S[:, 1] = rng.integers(0, 1 << 32, S.shape[0], dtype=np.uint64)
    want = oracle.join("phj_radix_lp", R, S)
    seg, exact = both(hj, cuda, "phj_radix_lp", R, S)
    assert (seg.matched_cnt, seg.checksum) == want == (exact.matched_cnt, exact.checksum)
    assert seg.large_partitions > 0


def test_segment_mode_materialising(hj, oracle, cuda):
    R, S = hj.gen_pkfk_uniform(1 << 14, 1 << 16, payload=True)
    want = oracle.join("phj_radix_bc", R, S)
    r = hj.join_mat("ptr_phj_radix_bc", R, S, flags=hj.HJ_F_SEGMENTS)
    assert (r.matched_cnt, r.checksum) == want


def test_segment_mode_by_size(hj, cuda):
    # From 2^27 tuples segment mode is the default; the exact pipeline gives the same result.
    nR, nS = 1 << 25, 1 << 27
    torch = cuda
    R = torch.empty((nR, 2), dtype=torch.int64, device="cuda")
    S = torch.empty((nS, 2), dtype=torch.int64, device="cuda")
    hj.gen_fast_device(nR, nS, R.data_ptr(), S.data_ptr(), seed=99)
    torch.cuda.synchronize()
    want = hj.pkfk_closed_form(nR, nS)
    d = hj.join("phj_radix_bc", R, S, on_device=True, flags=hj.HJ_F_PHASE_TIMES)
    e = hj.join("phj_radix_bc", R, S, on_device=True, flags=hj.HJ_F_EXACT | hj.HJ_F_PHASE_TIMES)
    assert (d.matched_cnt, d.checksum) == want == (e.matched_cnt, e.checksum)
    assert d.phase[0] == 0.0 and e.phase[0] > 0.0
    del R, S
    torch.cuda.empty_cache()


def test_segment_mode_stall_is_reported(hj, cuda):
    # The test hook withholds the first tile load of pass-1 CTA 0: its bounded wait expires, the join
    # returns HJ_E_TIMEOUT, and the context joins correctly afterwards. The relations have many more
    # tiles than there are pass-1 CTAs, so CTA 0 surely claims a tile.
    nR, nS = 1 << 20, 1 << 22
    torch = cuda
    R = torch.empty((nR, 2), dtype=torch.int64, device="cuda")
    S = torch.empty((nS, 2), dtype=torch.int64, device="cuda")
    hj.gen_fast_device(nR, nS, R.data_ptr(), S.data_ptr(), seed=5)
    torch.cuda.synchronize()
    ctx = hj.Context(0)
    try:
        r = hj.join("phj_radix_bc", R, S, on_device=True, ctx=ctx,
                    flags=hj.HJ_F_SEGMENTS | hj.HJ_F_TEST_STALL, check=False)
        assert r.status == hj.HJ_E_TIMEOUT
        r = hj.join("phj_radix_bc", R, S, on_device=True, ctx=ctx, flags=hj.HJ_F_SEGMENTS)
        assert (r.matched_cnt, r.checksum) == hj.pkfk_closed_form(nR, nS)
    finally:
        ctx.close()
