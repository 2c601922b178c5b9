"""Join server on the B200: every request's result equals the same join run alone (hj_join) and the
oracle, whichever implementation served it and whatever ran beside it; admission keeps the pool
within its budget; requests that can never fit are refused at submission."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ALGOS = ["nphj_sc", "nphj_lp", "phj_radix_bc", "phj_radix_lp"]


def _requests(seed, n, max_log=18):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nR = int(2 ** rng.uniform(3, max_log))
        nS = int(nR * rng.integers(1, 9))
        R = np.empty((nR, 2), dtype=np.uint64)
        S = np.empty((nS, 2), dtype=np.uint64)
        kr = nR if i % 3 else max(nR // 4, 1)  # every third request has duplicate build keys
        R[:, 0] = rng.integers(0 if i % 5 == 0 else 1, kr + 1, nR, dtype=np.uint64)  # some have key 0
        R[:, 1] = rng.integers(0, 2**40, nR, dtype=np.uint64)
        S[:, 0] = rng.integers(0 if i % 5 == 0 else 1, kr + kr // 3 + 2, nS, dtype=np.uint64)
        S[:, 1] = rng.integers(0, 2**40, nS, dtype=np.uint64)
        if i % 7 == 0:
            R[::13, 0] = np.uint64(2**64 - 1)
            S[::17, 0] = np.uint64(2**64 - 1)
        out.append((ALGOS[i % 4], R, S))
    return out


@pytest.mark.parametrize("slots,tuner,waves", [
    (8, None, True),
    (3, {"nphj_max_table_bytes": 1e6, "partition_target": 512, "wave_table_bytes": 64e6}, True),
    (1, None, True),
    (8, None, False),
    (2, {"nphj_max_table_bytes": 1e6, "partition_target": 512, "wave_table_bytes": 4e6}, True)])
def test_server_mix_matches_alone(hj, oracle, cuda, slots, tuner, waves):
    reqs = _requests(11 + slots, 48)
    alone = [hj.join(a, R, S) for a, R, S in reqs]
    dev = [(cuda.from_numpy(R.view(np.int64)).cuda(), cuda.from_numpy(S.view(np.int64)).cuda())
           for _, R, S in reqs]
    with hj.Server(0, slots=slots, hbm_budget_bytes=2e9, tuner=tuner, waves=waves) as srv:
        ids = {}
        for rep in range(2):
            for i, (a, R, S) in enumerate(reqs):
                on_dev = (i + rep) % 2 == 1
                rid = srv.submit(a, dev[i][0], dev[i][1], on_device=True) if on_dev else srv.submit(a, R, S)
                ids[rid] = i
                if i % 5 == 0:
                    time.sleep(0.0005)
        got = srv.wait_all(ids.keys())
        impls = set()
        for rid, c in got.items():
            i = ids[rid]
            a, R, S = reqs[i]
            assert c.status == 0, (a, R.shape, S.shape)
            assert (c.matched_cnt, c.checksum) == (alone[i].matched_cnt, alone[i].checksum), (a, R.shape, S.shape, c.impl)
            assert (c.matched_cnt, c.checksum) == oracle.join(a, R, S)
            assert c.submit_s <= c.start_s <= c.done_s
            impls.add(c.impl)
            if waves and c.impl == 0 and R.shape[0] and S.shape[0]:
                assert c.wave > 0 and c.wave_size >= 1  # non-partitioned requests run in waves
            else:
                assert c.wave == 0
        st = srv.stats()
        assert st.completed == st.submitted == 2 * len(reqs)
        assert st.in_use_bytes == 0 and st.queued == 0 and st.inflight == 0
        if waves:
            assert st.waves > 0 and st.wave_requests == sum(1 for c in got.values() if c.wave)
    if tuner:
        assert impls == {0, 1}


def test_server_waves_coalesce_a_burst(hj, oracle, cuda):
    """A burst of small requests submitted at once is served in a few waves of many requests each, and
    every result equals the same join alone and the oracle, whichever wave carried it."""
    reqs = _requests(97, 300, max_log=12)
    dev = [(cuda.from_numpy(R.view(np.int64)).cuda(), cuda.from_numpy(S.view(np.int64)).cuda())
           for _, R, S in reqs]
    with hj.Server(0, slots=4, hbm_budget_bytes=4e9, wave_max_requests=128) as srv:
        ids = {srv.submit(a, dev[i][0], dev[i][1], on_device=True): i for i, (a, R, S) in enumerate(reqs)}
        got = srv.wait_all(ids.keys())
        sizes = {}
        for rid, c in got.items():
            a, R, S = reqs[ids[rid]]
            assert c.status == 0
            assert (c.matched_cnt, c.checksum) == oracle.join(a, R, S), (a, R.shape, S.shape, c.wave)
            if c.wave:
                sizes[c.wave] = c.wave_size
        st = srv.stats()
    assert max(sizes.values()) > 1                      # requests were coalesced
    assert max(sizes.values()) <= 128                   # within the configured wave size
    assert st.waves == len(sizes) < st.wave_requests    # fewer waves than requests
    assert st.in_use_bytes == 0


def test_server_wave_shrinks_under_memory_pressure(hj, cuda):
    """With a pool that holds only a few requests' tables, waves shrink to what fits and every request
    is still served exactly (no wave waits forever for a block larger than the pool)."""
    nR, nS = 1 << 16, 1 << 18
    R, S = hj.gen_fast_host(nR, nS, seed=9)
    Rd = cuda.from_numpy(R.view(np.int64)).cuda()
    Sd = cuda.from_numpy(S.view(np.int64)).cuda()
    want = hj.pkfk_closed_form(nR, nS)
    with hj.Server(0, slots=2, hbm_budget_bytes=8e6) as srv:  # ~2.1 MB per request's table
        ids = [srv.submit("nphj_sc", Rd, Sd, on_device=True) for _ in range(40)]
        got = srv.wait_all(ids)
        assert all((c.status, c.matched_cnt, c.checksum) == (0, *want) for c in got.values())
        st = srv.stats()
        assert 0 < st.peak_in_use_bytes <= st.budget_bytes
        assert st.wave_requests == 40 and st.in_use_bytes == 0


def test_server_budget_admission(hj, cuda):
    # Each request needs ~11.5 MB (a 2 MB table plus its host relations copied into the pool); the pool
    # holds four at a time.
    nR, nS = 1 << 16, 1 << 19
    R, S = hj.gen_fast_host(nR, nS, seed=5)
    want = hj.pkfk_closed_form(nR, nS)
    budget = 56e6
    with hj.Server(0, slots=8, hbm_budget_bytes=budget) as srv:
        ids = [srv.submit("phj_radix_bc", R, S) for _ in range(24)]
        got = srv.wait_all(ids)
        assert all((c.status, c.matched_cnt, c.checksum) == (0, *want) for c in got.values())
        st = srv.stats()
        assert 0 < st.peak_in_use_bytes <= st.budget_bytes <= budget
        with pytest.raises(hj.JoinError) as e:
            big_R, big_S = hj.gen_fast_host(1 << 20, 1 << 21, seed=1)
            srv.submit("phj_radix_bc", big_R, big_S)
        assert e.value.status == hj.HJ_E_BUDGET


def test_server_degenerate_requests(hj, cuda):
    e = np.zeros((0, 2), dtype=np.uint64)
    one = np.array([[5, 50]], dtype=np.uint64)
    reqs = [("phj_radix_bc", e, one), ("nphj_sc", one, e), ("nphj_lp", one, one), ("phj_radix_lp", one, one),
            ("phj_radix_lp", np.array([[0, 7]], dtype=np.uint64), np.array([[0, 9]], dtype=np.uint64))]
    with hj.Server(0, slots=2, hbm_budget_bytes=1e8) as srv:
        ids = [srv.submit(a, R, S) for a, R, S in reqs]
        got = srv.wait_all(ids)
        assert [(got[i].matched_cnt, got[i].checksum) for i in ids] == [(0, 0), (0, 0), (1, 100), (1, 100), (0, 0)]


def test_server_invalid_arguments(hj, cuda):
    with pytest.raises(hj.JoinError):
        hj.Server(0, slots=0)
    with hj.Server(0, slots=1, hbm_budget_bytes=1e8) as srv:
        L = hj._bind_server()
        assert L.hj_server_submit(srv.handle, 7, None, 0, None, 0, 0, None) == hj.HJ_E_INVAL
        assert L.hj_server_submit(srv.handle, 0, None, 4, None, 0, 0, None) == hj.HJ_E_INVAL
