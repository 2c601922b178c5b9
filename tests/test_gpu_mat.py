"""Materialising joins (the reference's ptr_* joins) on the B200: the pairs written equal the oracle's
pair set, the retrieve checksum equals the reference's definition, and the buffer rules hold."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ALGOS = ["nphj_sc", "nphj_lp", "phj_radix_bc", "phj_radix_lp", "phj_radix_hr", "phj_asymm_radix_sc"]
U64MAX = np.uint64(2**64 - 1)


def positions(n):
    return np.arange(1, n + 1, dtype=np.uint64)


def dup_data(seed, nR, nS, key_range, zero=True, ones=True):
    rng = np.random.default_rng(seed)
    R = np.empty((nR, 2), dtype=np.uint64)
    S = np.empty((nS, 2), dtype=np.uint64)
    R[:, 0] = rng.integers(0 if zero else 1, key_range, nR, dtype=np.uint64)
    S[:, 0] = rng.integers(0 if zero else 1, key_range + key_range // 4, nS, dtype=np.uint64)
    if ones:
        R[::211, 0] = U64MAX
        S[::97, 0] = U64MAX
    R[:, 1] = positions(nR)
    S[:, 1] = positions(nS)
    return R, S


def sorted_pairs(P):
    P = np.asarray(P, dtype=np.uint64).reshape(-1, 2)
    return P[np.lexsort((P[:, 1], P[:, 0]))]


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


@pytest.mark.parametrize("algo", ALGOS)
def test_pairs_equal_oracle(hj, oracle, cuda, algo):
    R, S = dup_data(3, 20_000, 60_000, 9_000)
    want = oracle.join_pairs(algo, R, S)
    ref = oracle.join(algo.replace("asymm_radix", "radix"), R, S)
    # device buffers
    out = cuda.zeros((want.shape[0] + 10, 2), dtype=cuda.int64, device="cuda")
    r = hj.join_mat(algo, dev(cuda, R), dev(cuda, S), pairs=out, on_device=True, bits=12)
    assert r.matched_cnt == want.shape[0] == ref[0]
    assert r.checksum == ref[1]  # row ids are positions: the retrieve sum is the join's checksum
    got = sorted_pairs(out[: r.matched_cnt].cpu().numpy().view(np.uint64))
    assert np.array_equal(got, want)
    # host buffers
    hostp = np.zeros((want.shape[0], 2), dtype=np.uint64)
    r = hj.join_mat(algo, R, S, pairs=hostp, bits=14)
    assert (r.matched_cnt, r.checksum) == ref
    assert np.array_equal(sorted_pairs(hostp), want)
    # library-owned pairs (more matches than probe tuples for the every-match joins: one rerun)
    r = hj.join_mat("ptr_" + algo if not algo.startswith("phj_asymm") else algo, R, S)
    assert (r.matched_cnt, r.checksum) == ref
    assert r.total >= r.retrieve > 0


def test_capacity_and_row_id_errors(hj, oracle, cuda):
    R, S = dup_data(4, 5_000, 20_000, 1_000, zero=False, ones=False)
    need = oracle.join("phj_radix_bc", R, S)[0]
    small = np.zeros((need // 2, 2), dtype=np.uint64)
    r = hj.join_mat("phj_radix_bc", R, S, pairs=small, check=False)
    assert r.status == hj.HJ_E_CAPACITY and r.matched_cnt == need
    R2 = R.copy()
    R2[7, 1] = np.uint64(10**9)  # not a position of R
    r = hj.join_mat("phj_radix_bc", R2, S, check=False)
    assert r.status == hj.HJ_E_ROWID


def test_pkfk_payload_closed_form_and_large_partitions(hj, oracle, cuda):
    # payload PK-FK data (the reference's ptr_* workload): checksum |S|(|S|+1)/2 + m n(n+1)/2
    nR, nS = 1 << 16, 1 << 18
    R, S = hj.gen_pkfk_uniform(nR, nS, payload=True)
    m = nS // nR
    want = (nS, (nS * (nS + 1) // 2 + m * nR * (nR + 1) // 2) % 2**64)
    for algo in ("phj_radix_bc", "phj_radix_lp", "nphj_sc", "nphj_lp"):
        assert (lambda r: (r.matched_cnt, r.checksum))(hj.join_mat(algo, R, S)) == want, algo
    # 2 radix bits over 2^16 build tuples (16384 per partition, above the 10240 of the shared-memory
    # joins): every partition takes the global-memory path
    r = hj.join_mat("phj_radix_bc", R, S, bits=2, passes=1)
    assert (r.matched_cnt, r.checksum) == want and r.large_partitions > 0
    rd, sd = dup_data(5, 40_000, 80_000, 30_000)
    for algo in ("phj_radix_bc", "phj_radix_lp"):
        out = np.zeros((oracle.join_pairs(algo, rd, sd).shape[0], 2), dtype=np.uint64)
        r = hj.join_mat(algo, rd, sd, pairs=out, bits=1, passes=1)
        assert r.large_partitions > 0
        assert np.array_equal(sorted_pairs(out), oracle.join_pairs(algo, rd, sd))


def test_empty_relations(hj, cuda):
    e = np.zeros((0, 2), dtype=np.uint64)
    one = np.array([[5, 1]], dtype=np.uint64)
    for algo in ("phj_radix_bc", "nphj_lp"):
        r = hj.join_mat(algo, e, one)
        assert (r.matched_cnt, r.checksum) == (0, 0)
        r = hj.join_mat(algo, one, one)
        assert (r.matched_cnt, r.checksum) == (1, 2)
