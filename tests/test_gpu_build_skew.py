"""Build-side skew on the B200: partitions whose build side is far beyond the shared-memory tables,
with hot build keys (many build tuples sharing one key). The reference splits such partitions across
threads (SKEW_HANDLING, src/algo/phj.c:1374-1614) and still walks one chain entry per build tuple for
every probe; here joins that need no per-match output aggregate equal build keys (count, row-id sum,
first position), so each probe costs one lookup. Every result is checked against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def hot_build(rng, n_build, n_probe, part=5, bits=14, hot=(7, 11, 13), hot_share=0.9, key_space=1 << 20):
    """Every build key in radix partition `part` (low `bits` bits); `hot_share` of the build tuples
    carry one of the `hot` keys, the rest are spread over key_space keys. Probes: a quarter hot keys,
    the rest spread (some missing)."""
    R = np.empty((n_build, 2), dtype=np.uint64)
    is_hot = rng.random(n_build) < hot_share
    hi = np.where(is_hot, rng.choice(np.array(hot, dtype=np.uint64), n_build),
                  rng.integers(100, key_space, n_build, dtype=np.uint64))
    R[:, 0] = (hi << np.uint64(bits)) | np.uint64(part)
    R[:, 1] = rng.integers(0, 2**62, n_build, dtype=np.uint64)
    S = np.empty((n_probe, 2), dtype=np.uint64)
    shi = np.where(rng.random(n_probe) < 0.25, rng.choice(np.array(hot, dtype=np.uint64), n_probe),
                   rng.integers(100, key_space + key_space // 8, n_probe, dtype=np.uint64))
    S[:, 0] = (shi << np.uint64(bits)) | np.uint64(part)
    S[:, 1] = rng.integers(0, 2**62, n_probe, dtype=np.uint64)
    return R, S


@pytest.mark.parametrize("algo", ["phj_radix_bc", "phj_radix_lp"])
def test_hot_build_keys_in_one_giant_partition(hj, oracle, cuda, algo):
    """2^24 build tuples in one partition, 90% of them on three keys, 2^22 probes (a quarter hot):
    about 3.4e12 matching pairs, counted exactly in one lookup per probe."""
    rng = np.random.default_rng(5)
    R, S = hot_build(rng, 1 << 24, 1 << 22)
    want = oracle.join(algo, R, S)
    got = hj.join(algo, dev(cuda, R), dev(cuda, S), on_device=True, bits=14, passes=2)
    assert (got.matched_cnt, got.checksum) == want
    assert got.large_partitions >= 1
    if algo == "phj_radix_bc":
        assert got.matched_cnt > 10**12


def test_hot_build_keys_segment_mode_and_one_pass(hj, oracle, cuda):
    """The same giant hot partition through segment mode (pass 1 without offsets) and through a one-pass
    geometry, against the oracle; plus partitions of every size around the shared-memory limit."""
    rng = np.random.default_rng(6)
    R, S = hot_build(rng, 1 << 22, 1 << 23, part=77)
    want = oracle.join("phj_radix_bc", R, S)
    for flags, bits, passes in ((hj.HJ_F_SEGMENTS, 14, 2), (0, 14, 2), (0, 8, 1)):
        pr = (R[:, 0] & np.uint64((1 << bits) - 1)) == np.uint64(77 & ((1 << bits) - 1))
        assert pr.all()
        got = hj.join("phj_radix_bc", dev(cuda, R), dev(cuda, S), on_device=True, bits=bits, passes=passes,
                      flags=flags)
        assert (got.matched_cnt, got.checksum) == want, (flags, bits, passes)


@pytest.mark.parametrize("algo", ["phj_radix_bc", "phj_radix_lp", "phj_radix_sc"])
def test_many_large_partitions_mixed_sizes(hj, oracle, cuda, algo):
    """Dozens of partitions above the shared-memory limit with duplicate-heavy keys next to ordinary
    ones, key 0 included (the lp rule ignores it)."""
    rng = np.random.default_rng(8)
    n = 1 << 21
    R = np.empty((n, 2), dtype=np.uint64)
    part = rng.integers(0, 40, n, dtype=np.uint64)  # 40 partitions of ~52K build tuples
    R[:, 0] = (rng.integers(0, 3000, n, dtype=np.uint64) << np.uint64(12)) | part
    R[:, 1] = np.arange(n, dtype=np.uint64)
    S = R[rng.integers(0, n, 3 * n)].copy()
    S[:, 1] = rng.integers(0, 2**40, S.shape[0], dtype=np.uint64)
    S[::11, 0] += np.uint64(1 << 30)
    want = oracle.join(algo, R, S)
    got = hj.join(algo, dev(cuda, R), dev(cuda, S), on_device=True, bits=12, passes=2)
    assert (got.matched_cnt, got.checksum) == want
    assert got.large_partitions >= 30


def test_materialising_join_keeps_per_match_chains(hj, oracle, cuda):
    """ptr_ joins write one pair per match, so their large partitions keep per-tuple chains; the pairs
    equal the oracle's."""
    rng = np.random.default_rng(9)
    R, S = hot_build(rng, 30_000, 4_000, hot=(3,), hot_share=0.01, key_space=20_000)
    R[:, 1] = np.arange(1, R.shape[0] + 1, dtype=np.uint64)  # retrieve needs row id = position
    S[:, 1] = np.arange(1, S.shape[0] + 1, dtype=np.uint64)
    pairs_want = oracle.join_pairs("phj_radix_bc", R, S)
    cap = pairs_want.shape[0] + 16
    pairs = cuda.zeros((cap, 2), dtype=cuda.int64, device="cuda")
    r = hj.join_mat("ptr_phj_radix_bc", dev(cuda, R), dev(cuda, S), pairs=pairs, on_device=True)
    assert (r.matched_cnt, r.checksum) == oracle.join("phj_radix_bc", R, S)
    got = pairs[: r.matched_cnt].cpu().numpy().view(np.uint64)
    got = got[np.lexsort((got[:, 1], got[:, 0]))]
    assert np.array_equal(got, pairs_want)
