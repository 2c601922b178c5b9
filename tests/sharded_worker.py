"""Worker for test_sharded.py: one rank of a gloo process group (CPU) running the library's sharded
join plumbing (hashjoin_scm_b200.sharded_join): owner routing, the all-to-all of counts and of tuples,
the local joins and the all-reduce of the results. Routing and the local join are the oracle's host
restatements here (a CPU rank has no GPU); the exchange is real. Every rank checks the global result
against the oracle on the concatenation of all ranks' relations, and checks that the tuples it holds
after the exchange are exactly those it owns."""
import datetime
import importlib.util
import json
import os
import pathlib
import sys

import numpy as np
import torch
import torch.distributed as dist

ROOT = pathlib.Path(__file__).resolve().parents[1]


def load(name, path):
    spec = importlib.util.spec_from_file_location(name, path, submodule_search_locations=[str(path.parent)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


hj = load("hashjoin_scm_b200", ROOT / "hashjoin-scm_b200" / "__init__.py")
orc = load("hj_oracle", ROOT / "oracle" / "hj_oracle.py")


def relations(rank, nR, nS):
    """Rank-local relations over one shared key space: duplicate build keys, key 0, misses."""
    rng = np.random.default_rng(1000 + rank)
    R = np.empty((nR, 2), dtype=np.uint64)
    S = np.empty((nS, 2), dtype=np.uint64)
    R[:, 0] = rng.integers(0, 5000, nR, dtype=np.uint64)
    R[:, 1] = rng.integers(0, 2**63, nR, dtype=np.uint64)
    S[:, 0] = rng.integers(0, 6000, nS, dtype=np.uint64)
    S[:, 1] = rng.integers(0, 2**63, nS, dtype=np.uint64)
    return R, S


def as_tensor(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64))


def route(T, nshards):
    routed, counts = orc.shard_route(T.numpy().view(np.uint64), nshards)
    return as_tensor(routed), torch.from_numpy(counts)


held = {}


def local_join(algo, R, S):
    Rn, Sn = R.numpy().view(np.uint64), S.numpy().view(np.uint64)
    held[algo] = (Rn.copy(), Sn.copy())
    return orc.join(algo, Rn, Sn)


rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
sizes = [(3000 + 700 * r, 9000 + 1100 * r) for r in range(world)]
rels = [relations(r, *sizes[r]) for r in range(world)]
R_all = np.concatenate([r for r, _ in rels])
S_all = np.concatenate([s for _, s in rels])
out = {}
for algo in ("phj_radix_bc", "phj_radix_lp", "nphj_sc", "nphj_lp"):
    got = hj.sharded_join(algo, as_tensor(rels[rank][0]), as_tensor(rels[rank][1]), route=route,
                          local_join=local_join)
    want = orc.join(algo, R_all, S_all)
    assert got == want, (rank, algo, got, want)
    # This rank holds exactly the tuples it owns, build side in global input order.
    Rh, Sh = held[algo]
    own_R = R_all[orc.shard_of(R_all[:, 0], world) == rank]
    own_S = S_all[orc.shard_of(S_all[:, 0], world) == rank]
    assert np.array_equal(Rh, own_R) and np.array_equal(Sh, own_S), (rank, algo)
    out[algo] = [int(got[0]), int(got[1])]
dist.barrier()
if rank == 0:
    print(json.dumps({"world": world, "results": out}), flush=True)
dist.destroy_process_group()
