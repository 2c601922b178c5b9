"""bench.py's N > 1 path on CPU: two gloo ranks launched by torchrun, as the driver launches the bench
(one rank per GPU there). Checks the max over ranks, the weak-scaling whole-job value, that only rank 0
prints, and that non-zero ranks of the reference arm exit without work."""
import json
import os
import pathlib
import socket
import subprocess
import sys

ROOT = pathlib.Path(__file__).resolve().parents[1]


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           str(ROOT / "tests" / "multirank_worker.py")]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=240, env=env)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-4000:]
    lines = [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    ln = lines[0]
    assert ln["ms"] == 11.0                      # the slowest rank
    assert ln["value"] == 2 * 3000 / 0.011       # all ranks' tuples over the slowest time
    assert ln["serve"] == 2 * 100.0              # the slowest rank's rate, times the ranks
    assert ln["n_gpus"] == 2
