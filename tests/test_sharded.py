"""Sharded joins across ranks: the exchange plumbing on CPU-only gloo process groups (2 and 3 ranks,
launched by torchrun as the GPU runs are), the oracle's owner function against the library's routing
kernel (GPU), and a one-rank NCCL run of the whole device path (routing kernel, all-to-all, GPU join,
all-reduce)."""
import json
import os
import pathlib
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_join_exchange_on_gloo_ranks(oracle, world):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={world}",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           str(ROOT / "tests" / "sharded_worker.py")]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-4000:]
    lines = [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1 and lines[0]["world"] == world
    assert set(lines[0]["results"]) == {"phj_radix_bc", "phj_radix_lp", "nphj_sc", "nphj_lp"}


def test_owner_function_spreads_keys(oracle):
    keys = np.arange(1, 1 << 20, dtype=np.uint64)
    for n in (1, 2, 3, 8, 32):
        own = oracle.shard_of(keys, n)
        assert own.min() >= 0 and own.max() < n
        counts = np.bincount(own, minlength=n)
        assert counts.max() - counts.min() < 0.02 * keys.size / n + 64


@pytest.mark.gpu
@pytest.mark.parametrize("n,nshards", [(0, 2), (1, 3), (5000, 2), (1 << 20, 8), ((1 << 22) + 17, 5), (3000, 32)])
def test_route_kernel_matches_oracle(hj, oracle, cuda, n, nshards):
    rng = np.random.default_rng(n + nshards)
    T = np.empty((n, 2), dtype=np.uint64)
    T[:, 0] = rng.integers(0, 2**64 - 1, n, dtype=np.uint64)
    T[: n // 3, 0] = rng.integers(0, 100, n // 3, dtype=np.uint64)  # repeated keys
    T[:, 1] = np.arange(n, dtype=np.uint64)
    Td = cuda.from_numpy(T.view(np.int64)).cuda()
    routed, counts = hj.shard_route(Td, nshards)
    cuda.cuda.synchronize()
    want, want_counts = oracle.shard_route(T, nshards)
    assert np.array_equal(counts.cpu().numpy(), want_counts)
    assert np.array_equal(routed.cpu().numpy().view(np.uint64), want)


_NCCL_ONE_RANK = r"""
import datetime, importlib.util, json, pathlib, sys
import numpy as np, torch, torch.distributed as dist
root = pathlib.Path(sys.argv[1])
def load(name, path):
    spec = importlib.util.spec_from_file_location(name, path, submodule_search_locations=[str(path.parent)])
    m = importlib.util.module_from_spec(spec); sys.modules[name] = m; spec.loader.exec_module(m); return m
hj = load("hashjoin_scm_b200", root / "hashjoin-scm_b200" / "__init__.py")
orc = load("hj_oracle", root / "oracle" / "hj_oracle.py")
torch.cuda.set_device(0)
dist.init_process_group("nccl", store=dist.HashStore(), rank=0, world_size=1,
                        timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
R, S = hj.gen_dup_uniform(1 << 14, 1 << 16)
Rd = torch.from_numpy(R.view(np.int64)).cuda(); Sd = torch.from_numpy(S.view(np.int64)).cuda()
res = {}
for algo in ("phj_radix_bc", "phj_radix_lp", "nphj_sc", "nphj_lp"):
    got = hj.sharded_join(algo, Rd, Sd)
    assert got == orc.join(algo, R, S), (algo, got)
    res[algo] = list(got)
dist.destroy_process_group()
print(json.dumps(res))
"""


@pytest.mark.gpu
def test_sharded_join_device_path_one_rank(hj, cuda):
    out = subprocess.run([sys.executable, "-c", _NCCL_ONE_RANK, str(ROOT)], capture_output=True, text=True,
                         timeout=300, env=dict(os.environ, NCCL_NVLS_ENABLE="0"))
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-4000:]
    assert json.loads(out.stdout.strip().splitlines()[-1])
