"""Streamed joins on the B200 (hj_join_streamed): R on the device, S in chunks from host memory; every
chunking gives hj_join's result, for every algorithm, including ragged last chunks and one chunk."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ALGOS = ["nphj_sc", "nphj_lp", "phj_radix_bc", "phj_radix_lp", "phj_radix_hr"]


@pytest.mark.parametrize("algo", ALGOS)
def test_streamed_equals_join(hj, oracle, cuda, algo):
    rng = np.random.default_rng(21)
    nR, nS = 50_000, 333_333
    R = np.empty((nR, 2), dtype=np.uint64)
    S = np.empty((nS, 2), dtype=np.uint64)
    R[:, 0] = rng.integers(0, 20_000, nR, dtype=np.uint64)  # duplicates: lp order matters
    S[:, 0] = rng.integers(0, 25_000, nS, dtype=np.uint64)
    R[:, 1] = rng.integers(0, 2**63, nR, dtype=np.uint64)
    S[:, 1] = rng.integers(0, 2**63, nS, dtype=np.uint64)
    R[::101, 0] = np.uint64(2**64 - 1)
    S[::103, 0] = np.uint64(2**64 - 1)
    want = oracle.join(algo, R, S)
    with hj.Context(0) as ctx:
        for chunk in (0, 1 << 16, 100_000, 7_777, nS):
            r = hj.join_streamed(algo, R, S, ctx, chunk_tuples=chunk, bits=12)
            assert (r.matched_cnt, r.checksum) == want, (algo, chunk)
        # the context's ordinary joins still work after a streamed one
        r = hj.join(algo, R, S, ctx=ctx)
        assert (r.matched_cnt, r.checksum) == want


def test_streamed_pkfk_and_arguments(hj, cuda):
    nR, nS = 1 << 18, 1 << 22
    R, S = hj.gen_fast_host(nR, nS, seed=4)
    with hj.Context(0) as ctx:
        r = hj.join_streamed("phj_radix_bc", R, S, ctx, chunk_tuples=1 << 20)
        assert (r.matched_cnt, r.checksum) == hj.pkfk_closed_form(nR, nS)
        assert r.total > 0
        e = np.zeros((0, 2), dtype=np.uint64)
        assert hj.join_streamed("nphj_sc", e, S, ctx).matched_cnt == 0
        assert hj.join_streamed("phj_radix_lp", R, e, ctx).matched_cnt == 0
        L = hj.lib()
        p = hj.make_params(on_device=True)
        res = hj.Result()
        assert L.hj_join_streamed(ctx.handle, 2, hj.ctypes.byref(p), R.ctypes.data, nR, S.ctypes.data, nS, 0,
                                  hj.ctypes.byref(res)) == hj.HJ_E_INVAL  # device relations: not for this entry
