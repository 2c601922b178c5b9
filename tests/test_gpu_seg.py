"""GPU parity of segment mode: the radix joins that count every match partition in pass 1 into
chains of fixed-size segments and count the histograms on the way (no histogram pass). Forced at
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


def test_segment_mode_not_for_first_match(hj, oracle, cuda):
    # phj_radix_lp depends on input order within partitions: the flag leaves it on the exact pipeline.
    rng = np.random.default_rng(8)
    R = random_rel(rng, 40_000, 1, 10_000)
    S = random_rel(rng, 90_000, 1, 12_000)
    seg, exact = both(hj, cuda, "phj_radix_lp", R, S)
    want = oracle.join("phj_radix_lp", R, S)
    assert (seg.matched_cnt, seg.checksum) == want == (exact.matched_cnt, exact.checksum)
    assert seg.phase[0] > 0.0  # the histogram pass ran


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
