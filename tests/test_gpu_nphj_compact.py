"""GPU parity of the non-partitioned join's two slot layouts. When its 16-byte table would exceed 64 MB
(over 2^21 build tuples), nphj_sc and nphj_lp pack a build tuple into one 8-byte slot if every build key
is below 2^32 - 1 and every build row id below 2^32, and use 16-byte slots otherwise; both must give the
oracle's result bit for bit, at and around the limits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def rel(keys, rids):
    return np.stack([np.asarray(keys, dtype=np.uint64), np.asarray(rids, dtype=np.uint64)], axis=1)


def check(hj, oracle, cuda, R, S, algo="nphj_sc"):
    want = oracle.join(algo, R, S)
    r = hj.join(algo, dev(cuda, R), dev(cuda, S), on_device=True)
    assert (r.matched_cnt, r.checksum) == want, (algo, len(R), len(S))
    h = hj.join(algo, R, S)
    assert (h.matched_cnt, h.checksum) == want


def test_compact_slots_limits(hj, oracle, cuda):
    rng = np.random.default_rng(17)
    n = 1 << 22
    keys = rng.integers(1, 2**32 - 2, n, dtype=np.uint64)
    rids = rng.integers(0, 2**32, n, dtype=np.uint64)
    probe = np.concatenate([keys[rng.integers(0, n, n)], rng.integers(0, 2**64 - 1, n // 4, dtype=np.uint64)])
    S = rel(probe, rng.integers(0, 2**64 - 1, probe.size, dtype=np.uint64))
    # compact: largest key 2^32 - 2, largest row id 2^32 - 1
    k = keys.copy()
    k[0] = 2**32 - 2
    r = rids.copy()
    r[1] = 2**32 - 1
    check(hj, oracle, cuda, rel(k, r), S)
    # wide: one key equal to 2^32 - 1 (the compact empty pattern's key half)
    k2 = k.copy()
    k2[2] = 2**32 - 1
    S2 = S.copy()
    S2[:10, 0] = 2**32 - 1
    check(hj, oracle, cuda, rel(k2, r), S2)
    # wide: one row id of 2^32
    r2 = r.copy()
    r2[3] = 2**32
    check(hj, oracle, cuda, rel(k, r2), S)
    # wide: a build key of all ones (the 16-byte table's side record)
    k3 = k.copy()
    k3[4] = 2**64 - 1
    S3 = S.copy()
    S3[:7, 0] = 2**64 - 1
    check(hj, oracle, cuda, rel(k3, r), S3)


def test_compact_slots_duplicates(hj, oracle, cuda):
    # Duplicate build keys: every equal key counts, so probes walk to the empty slot.
    rng = np.random.default_rng(5)
    nR = 3 << 20
    R = rel(rng.integers(0, 1 << 20, nR), rng.integers(0, 2**32, nR))
    S = rel(rng.integers(0, 5 << 18, 1 << 20), rng.integers(0, 2**64 - 1, 1 << 20, dtype=np.uint64))
    check(hj, oracle, cuda, R, S)
    # nphj_lp: compact slots built by slices, one slot per key holding the first build tuple in input order
    check(hj, oracle, cuda, R, S, "nphj_lp")


def test_compact_slots_pkfk_sizes(hj, cuda):
    # The reference's CPU configuration, 2^22 x 2^23 (compact slots), and sizes on both sides of the
    # 64 MB limit.
    # (|S| a multiple of |R|: the closed form assumes every key occurs equally often in S.)
    for nR, nS in ((1 << 22, 1 << 23), ((1 << 21) + 5, 3 * ((1 << 21) + 5)), ((1 << 21) - 5, (1 << 21) - 5),
                   (1000, 3000)):
        R = cuda.empty((nR, 2), dtype=cuda.int64, device="cuda")
        S = cuda.empty((nS, 2), dtype=cuda.int64, device="cuda")
        hj.gen_fast_device(nR, nS, R.data_ptr(), S.data_ptr(), seed=31)
        cuda.cuda.synchronize()
        r = hj.join("nphj_sc", R, S, on_device=True)
        assert (r.matched_cnt, r.checksum) == hj.pkfk_closed_form(nR, nS)


def test_sliced_build_and_its_fallback(hj, oracle, cuda):
    """Compact tables are built slice by slice in shared memory (8192 slots per slice, probes wrap
    inside the slice) unless some slice would be filled above 7/8: then the build claims global slots by
    CAS instead. Both modes give the oracle's result: uniform keys (sliced), one key repeated 9000 times
    (its slice overfills: fallback), and a key repeated 2500 times (its slice holds ~6600 of 8192 slots:
    sliced, with a long cluster)."""
    rng = np.random.default_rng(23)
    nR = (1 << 21) + 4099
    base = rng.integers(1, 2**32 - 2, nR, dtype=np.uint64)
    rids = rng.integers(0, 2**32, nR, dtype=np.uint64)
    for hot in (0, 9000, 2500):
        k = base.copy()
        if hot:
            k[rng.choice(nR, hot, replace=False)] = np.uint64(123456789)
        nS = 3 << 20
        probe = k[rng.integers(0, nR, nS)]
        probe[::13] = rng.integers(1, 2**33, probe[::13].size, dtype=np.uint64)
        probe[::101] = np.uint64(123456789)
        S = rel(probe, rng.integers(0, 2**64 - 1, nS, dtype=np.uint64))
        check(hj, oracle, cuda, rel(k, rids), S)
        # first match: the sliced build keeps the first build tuple per key; the fallback is the 16-byte
        # table with its duplicate rebuild
        check(hj, oracle, cuda, rel(k, rids), S, "nphj_lp")
