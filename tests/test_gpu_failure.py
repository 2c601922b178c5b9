"""Failure detection on the B200 without a GPU fault: a bounded device wait that expires comes back
as HJ_E_TIMEOUT, the host watchdog gives up on a long join, and in both cases the context keeps
working for the next join (whose result is exact)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_device_wait_expires_and_context_recovers(hj, cuda):
    nR, nS = 1 << 20, 1 << 22
    R = cuda.empty((nR, 2), dtype=cuda.int64, device="cuda")
    S = cuda.empty((nS, 2), dtype=cuda.int64, device="cuda")
    hj.gen_fast_device(nR, nS, R.data_ptr(), S.data_ptr(), seed=9)
    cuda.cuda.synchronize()
    want = hj.pkfk_closed_form(nR, nS)
    with hj.Context(0) as ctx:
        assert (lambda r: (r.matched_cnt, r.checksum))(hj.join("phj_radix_bc", R, S, on_device=True, ctx=ctx)) == want
        t0 = time.time()
        # One CTA of the first partition pass never gets its tile: its wait gives up after ~2 s.
        r = hj.join("phj_radix_bc", R, S, on_device=True, ctx=ctx, flags=hj.HJ_F_TEST_STALL, check=False)
        assert r.status == hj.HJ_E_TIMEOUT
        assert 1.0 < time.time() - t0 < 60
        for algo in ("phj_radix_bc", "phj_radix_lp", "nphj_sc"):
            r = hj.join(algo, R, S, on_device=True, ctx=ctx)
            assert (r.matched_cnt, r.checksum) == want, algo


def test_host_watchdog(hj, cuda):
    nR, nS = 1 << 25, 1 << 27
    R = cuda.empty((nR, 2), dtype=cuda.int64, device="cuda")
    S = cuda.empty((nS, 2), dtype=cuda.int64, device="cuda")
    hj.gen_fast_device(nR, nS, R.data_ptr(), S.data_ptr(), seed=10)
    cuda.cuda.synchronize()
    want = hj.pkfk_closed_form(nR, nS)
    with hj.Context(0) as ctx:
        hj.join("phj_radix_bc", R, S, on_device=True, ctx=ctx)  # sizes the arena
        # A ~3 ms join against a 1 ms deadline: the call returns HJ_E_TIMEOUT while the join runs on.
        r = hj.join("phj_radix_bc", R, S, on_device=True, ctx=ctx, watchdog_ms=1, check=False)
        assert r.status == hj.HJ_E_TIMEOUT
        # The next call (another stream) waits for it and is exact.
        s2 = cuda.cuda.Stream()
        r = hj.join("phj_radix_bc", R, S, on_device=True, ctx=ctx, stream=s2.cuda_stream, watchdog_ms=60_000)
        assert (r.matched_cnt, r.checksum) == want
