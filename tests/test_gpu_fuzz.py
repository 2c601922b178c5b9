"""Randomised parity on the B200: many small joins of random shape -- sizes from 0 to ~50K, key
ranges from very dense (heavy duplication) to sparse (few matches), keys 0 and 2^64-1 mixed in,
radix bits 1..15 with one or two passes and random pass-1 splits, host or device inputs -- every
algorithm against the oracle, bit for bit; materialising joins against the oracle's pair set."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ALGOS = ["nphj_sc", "nphj_lp", "phj_radix_bc", "phj_radix_lp", "phj_radix_hr"]
U64MAX = np.uint64(2**64 - 1)


def random_case(rng):
    nR = int(rng.choice([0, 1, 2, int(rng.integers(3, 300)), int(rng.integers(300, 50_000))]))
    nS = int(rng.choice([0, 1, int(rng.integers(2, 500)), int(rng.integers(500, 60_000))]))
    key_range = int(rng.choice([2, 50, max(nR // 8, 1), max(nR, 1), 4 * max(nR, 1), 2**40]))
    key_range = max(key_range, nR * nS // 5_000_000 + 1)  # at most ~5M matches: chains stay short
    R = np.empty((nR, 2), dtype=np.uint64)
    S = np.empty((nS, 2), dtype=np.uint64)
    R[:, 0] = rng.integers(0, key_range, nR, dtype=np.uint64)
    S[:, 0] = rng.integers(0, key_range + key_range // 3 + 1, nS, dtype=np.uint64)
    if rng.random() < 0.3 and nR:
        R[rng.integers(0, nR, max(nR // 50, 1)), 0] = U64MAX
    if rng.random() < 0.3 and nS:
        S[rng.integers(0, nS, max(nS // 50, 1)), 0] = U64MAX
    if rng.random() < 0.5:  # row ids as positions (materialising joins need them)
        R[:, 1] = np.arange(1, nR + 1, dtype=np.uint64)
        S[:, 1] = np.arange(1, nS + 1, dtype=np.uint64)
        positions = True
    else:
        R[:, 1] = rng.integers(0, 2**64 - 1, nR, dtype=np.uint64)
        S[:, 1] = rng.integers(0, 2**64 - 1, nS, dtype=np.uint64)
        positions = False
    bits = int(rng.integers(1, 16))
    passes = int(rng.integers(1, 3))
    b1 = int(rng.integers(0, 9))
    return R, S, bits, passes, b1, positions


@pytest.mark.parametrize("seed", range(24))
def test_random_joins(hj, oracle, cuda, seed):
    rng = np.random.default_rng(1000 + seed)
    for _ in range(8):
        R, S, bits, passes, b1, positions = random_case(rng)
        on_dev = bool(rng.integers(0, 2))
        Rin = cuda.from_numpy(R.view(np.int64)).cuda() if on_dev else R
        Sin = cuda.from_numpy(S.view(np.int64)).cuda() if on_dev else S
        for algo in ALGOS:
            want = oracle.join(algo, R, S)
            r = hj.join(algo, Rin, Sin, on_device=on_dev, bits=bits, passes=passes, bits_pass1=b1)
            assert (r.matched_cnt, r.checksum) == want, (algo, R.shape, S.shape, bits, passes, b1, on_dev)
        if positions:
            algo = ALGOS[int(rng.integers(0, len(ALGOS)))]
            pairs = oracle.join_pairs(algo, R, S)
            out = np.zeros((pairs.shape[0] + 1, 2), dtype=np.uint64)
            r = hj.join_mat(algo, R, S, pairs=out, bits=bits, passes=passes, bits_pass1=b1)
            got = out[: r.matched_cnt]
            got = got[np.lexsort((got[:, 1], got[:, 0]))]
            assert np.array_equal(got, pairs), (algo, R.shape, S.shape, bits, passes)
            assert (r.matched_cnt, r.checksum) == oracle.join(algo, R, S)
