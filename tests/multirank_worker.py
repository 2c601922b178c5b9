"""Worker for test_multirank.py: one of WORLD_SIZE ranks (gloo on CPU) running bench.py's multi-rank
plumbing -- process-group set-up from the torchrun environment, max/min over ranks, the weak-scaling
aggregate, rank-0-only output and the reference arm's rank rule -- with per-rank numbers that stand in
for the device timings."""
import datetime
import importlib.util
import json
import os
import pathlib
import sys

import torch.distributed as dist

ROOT = pathlib.Path(__file__).resolve().parents[1]
spec = importlib.util.spec_from_file_location("bench", ROOT / "bench.py")
bench = importlib.util.module_from_spec(spec)
spec.loader.exec_module(bench)

rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
dev = "cpu"
# Rank r "took" 10 + r ms for 3 steps of 1000 tuples; rank r "served" 100 + r joins/s.
ms = bench.reduce_over_ranks(10.0 + rank, dist, dev)
slowest_rate = bench.reduce_over_ranks(100.0 + rank, dist, dev, op="min")
line = {"metric": "t", "value": bench.whole_job_rate(3 * 1000, world, ms / 1e3), "ms": ms,
        "serve": world * slowest_rate, "n_gpus": world}
dist.barrier()
bench.emit(rank, line)
# The reference arm runs on rank 0 only; the other ranks return at once, without any work.
if rank != 0:
    sys.argv = ["bench.py", "--impl", "reference"]
    assert bench.run_reference_arm(bench.parse_args(), rank, world) == 0
dist.barrier()
dist.destroy_process_group()
