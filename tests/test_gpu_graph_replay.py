"""Repeated device-resident joins on one context: the second identical call in a row is captured into a
CUDA graph and later ones replay it. Every call must still compute the join of what the buffers hold
now (the graph re-runs every kernel), with phase timings, across graph eviction and arena growth."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def rel(rng, n, kmax):
    a = np.empty((n, 2), dtype=np.uint64)
    a[:, 0] = rng.integers(1, kmax, n, dtype=np.uint64)
    a[:, 1] = rng.integers(0, 1 << 40, n, dtype=np.uint64)
    return a


@pytest.mark.parametrize("algo", ["nphj_sc", "phj_radix_bc", "phj_radix_lp", "nphj_lp"])
def test_replays_follow_the_buffers(hj, oracle, cuda, algo):
    rng = np.random.default_rng(31)
    R, S = rel(rng, 30_000, 50_000), rel(rng, 70_000, 60_000)
    dR, dS = dev(cuda, R), dev(cuda, S)
    with hj.Context(0) as ctx:
        want = oracle.join(algo, R, S)
        for i in range(4):  # plain, captured, replayed, replayed
            r = hj.join(algo, dR, dS, on_device=True, ctx=ctx, flags=hj.HJ_F_PHASE_TIMES)
            assert (r.matched_cnt, r.checksum) == want, i
            assert r.total > 0 and r.kernel_launches > 0
            assert sum(r.phase) > 0
        # new contents in the same buffers: the replay joins them
        R2, S2 = rel(rng, 30_000, 20_000), rel(rng, 70_000, 25_000)
        dR.copy_(dev(cuda, R2))
        dS.copy_(dev(cuda, S2))
        cuda.cuda.synchronize()
        r = hj.join(algo, dR, dS, on_device=True, ctx=ctx, flags=hj.HJ_F_PHASE_TIMES)
        assert (r.matched_cnt, r.checksum) == oracle.join(algo, R2, S2)


def test_many_keys_eviction_and_arena_growth(hj, oracle, cuda):
    rng = np.random.default_rng(32)
    pairs = [(rel(rng, 5_000 * (k + 1), 9_000), rel(rng, 12_000, 9_000)) for k in range(6)]
    dev_pairs = [(dev(cuda, R), dev(cuda, S)) for R, S in pairs]
    wants = [oracle.join("phj_radix_bc", R, S) for R, S in pairs]
    with hj.Context(0) as ctx:
        for rnd in range(3):
            for (dR, dS), want in zip(dev_pairs, wants):  # six keys: more than the graphs kept
                for _ in range(3):
                    r = hj.join("phj_radix_bc", dR, dS, on_device=True, ctx=ctx, flags=hj.HJ_F_NO_TIMING)
                    assert (r.matched_cnt, r.checksum) == want
            # a larger join grows the arena (the graphs are dropped), then the small ones again
            big_R, big_S = rel(rng, 400_000, 800_000), rel(rng, 900_000, 800_000)
            r = hj.join("nphj_sc", dev(cuda, big_R), dev(cuda, big_S), on_device=True, ctx=ctx)
            assert (r.matched_cnt, r.checksum) == oracle.join("nphj_sc", big_R, big_S)
