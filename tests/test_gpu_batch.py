"""Batched joins on the B200: every job's result equals the same join run alone (hj_join) and the
oracle, whichever implementation the autotuner picked, with and without the captured graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ALGOS = ["nphj_sc", "nphj_lp", "phj_radix_bc", "phj_radix_lp"]


def _jobs(cuda, seed, n_jobs):
    rng = np.random.default_rng(seed)
    jobs, host = [], []
    for i in range(n_jobs):
        nR = int(2 ** rng.uniform(4, 18))
        nS = int(nR * rng.integers(1, 9))
        R = np.empty((nR, 2), dtype=np.uint64)
        S = np.empty((nS, 2), dtype=np.uint64)
        kr = nR if i % 3 else max(nR // 4, 1)  # every third job has duplicate build keys
        R[:, 0] = rng.integers(0 if i % 5 == 0 else 1, kr + 1, nR, dtype=np.uint64)  # some have key 0
        R[:, 1] = rng.integers(0, 2**40, nR, dtype=np.uint64)
        S[:, 0] = rng.integers(0 if i % 5 == 0 else 1, kr + kr // 3 + 2, nS, dtype=np.uint64)
        S[:, 1] = rng.integers(0, 2**40, nS, dtype=np.uint64)
        if i % 7 == 0:
            R[::13, 0] = np.uint64(2**64 - 1)
            S[::17, 0] = np.uint64(2**64 - 1)
        algo = ALGOS[i % 4]
        Rd = cuda.from_numpy(R.view(np.int64)).cuda()
        Sd = cuda.from_numpy(S.view(np.int64)).cuda()
        jobs.append((algo, Rd, Sd))
        host.append((algo, R, S))
    return jobs, host


@pytest.mark.parametrize("mode", ["auto", "all_nphj", "all_phj", "small_waves"])
@pytest.mark.parametrize("graph", [True, False])
def test_batch_matches_single_joins(hj, oracle, cuda, mode, graph):
    jobs, host = _jobs(cuda, 3, 40)
    with hj.Context(0) as ctx:
        if mode == "all_nphj":
            hj.tuner_set(ctx, nphj_max_table_bytes=1e12)
        elif mode == "all_phj":
            hj.tuner_set(ctx, nphj_max_table_bytes=0.0, partition_target=512)
        elif mode == "small_waves":
            hj.tuner_set(ctx, nphj_max_table_bytes=1e12, wave_table_bytes=1e5)
        with hj.Batch(ctx, jobs, graph=graph) as b:
            for rep in range(2):
                res, st = b.run()
                assert st.nphj_jobs + st.phj_jobs == len(jobs)
                for (algo, R, S), r, (_, Rh, Sh) in zip(jobs, res, host):
                    assert r.status == 0
                    want = oracle.join(algo, Rh, Sh)
                    assert (r.matched_cnt, r.checksum) == want, (algo, R.shape, S.shape, r.impl, mode)
        if mode == "all_phj":
            assert st.phj_jobs == len(jobs)
        if mode == "all_nphj":
            assert st.nphj_jobs == len(jobs)


def test_tuner_decisions(hj, cuda):
    with hj.Context(0) as ctx:
        hj.tuner_set(ctx, nphj_max_table_bytes=64e6, partition_target=6144)
        L = hj._bind_batch()
        import ctypes
        impl, bits, passes = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        L.hj_tuner_decide(ctx.handle, 1 << 20, 1 << 23, ctypes.byref(impl), ctypes.byref(bits), ctypes.byref(passes))
        assert impl.value == 0
        L.hj_tuner_decide(ctx.handle, 1 << 27, 1 << 29, ctypes.byref(impl), ctypes.byref(bits), ctypes.byref(passes))
        assert impl.value == 1 and bits.value == 15 and passes.value == 2


def test_batch_empty_and_degenerate_jobs(hj, cuda):
    e = cuda.zeros((0, 2), dtype=cuda.int64, device="cuda")
    one = cuda.tensor([[5, 50]], dtype=cuda.int64, device="cuda")
    jobs = [("phj_radix_bc", e, one), ("nphj_sc", one, e), ("nphj_lp", one, one), ("phj_radix_lp", one, one)]
    with hj.Context(0) as ctx, hj.Batch(ctx, jobs) as b:
        res, _ = b.run()
        assert [(r.matched_cnt, r.checksum) for r in res] == [(0, 0), (0, 0), (1, 100), (1, 100)]


def test_batch_tuning_keeps_results(hj, oracle, cuda):
    # HJ_F_TUNE plans the batch under several table budgets and keeps the fastest plan; whichever it
    # keeps, every result is the oracle's and the tuner keeps the chosen budget.
    jobs, host = _jobs(cuda, 7, 30)
    with hj.Context(0) as ctx:
        before = hj.tuner_get(ctx).nphj_max_table_bytes
        with hj.Batch(ctx, jobs, tune=True) as b:
            res, st = b.run()
            for (algo, R, S), r, (_, Rh, Sh) in zip(jobs, res, host):
                assert r.status == 0 and (r.matched_cnt, r.checksum) == oracle.join(algo, Rh, Sh)
        after = hj.tuner_get(ctx).nphj_max_table_bytes
        assert after in [before * f for f in (1 / 32, 1 / 16, 0.125, 0.25, 0.5, 1.0, 2.0, 4.0)]
