#!/usr/bin/env python3
"""Benchmark of the B200 equi-join hot path (one JSON line on rank 0).

Workload (the headline configuration): phj_radix_bc, R = 2^27 and S = 2^29 tuples of 16 bytes
{int64 key, int64 row_id}; R keys a seeded permutation of 1..2^27, S holds every R key 4 times in
seeded order (the reference's gen_pkfk_uniform distribution, generated in parallel on the device);
14 radix bits in 2 passes. One step = one full join (histogram, two partition passes, partition
joins). Metric: (|R| + |S|) / join time, the reference's throughput definition (phases timed as
buildpart + probejoin, src/algo/phj.c:2509-2511).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own multithreaded CPU join (compiled from its sources into
oracle/_ref) on the host cores, on the same workload, and prints the same line with impl=reference.
With N > 1 (torchrun) every rank joins its own relations: independent joins, no collective on the
data path (weak scaling); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
PKG_DIR = ROOT / "hashjoin-scm_b200"
METRIC = "join throughput (|R|+|S|)/s and % HBM roofline at 1 B200; batched joins/s; p99"
UNIT = "tuples/s"
FALLBACK_HBM_GBS = 6650.0


def load_module(name, path):
    spec = importlib.util.spec_from_file_location(name, path, submodule_search_locations=[str(path.parent)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", choices=["join", "batch", "serve", "skew", "mat", "stream"], default="join",
                    help="join: the headline 2^27 x 2^29 join; batch: 512 independent joins; "
                         "serve: a Poisson stream of join requests through the join server; "
                         "skew: 2^26 x 2^28 lp joins on Zipf and duplicate-key data; "
                         "mat: the materialising ptr_ join at the headline size; "
                         "stream: R on the device, 2^32 probe tuples streamed from host memory")
    ap.add_argument("--rates", default="250,1000,2000,3000",
                    help="serve mode: offered request rates (requests/s) to sweep")
    ap.add_argument("--requests", type=int, default=1000, help="serve mode: requests per rate")
    ap.add_argument("--slots", type=int, default=8, help="serve mode: concurrent requests on the GPU")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serve mode: HBM pool budget")
    ap.add_argument("--large-share", type=float, default=None,
                    help="serve mode: SM share of large requests' kernels (default: the library's)")
    ap.add_argument("--batch-jobs", type=int, default=512)
    ap.add_argument("--calibrate", action="store_true",
                    help="batch mode: tune the batch plan on the device first (HJ_F_TUNE)")
    ap.add_argument("--algo", default="phj_radix_bc")
    ap.add_argument("--nr-log", type=int, default=27)
    ap.add_argument("--ns-log", type=int, default=29)
    ap.add_argument("--bits", type=int, default=14)
    ap.add_argument("--passes", type=int, default=2)
    ap.add_argument("--pipeline", choices=["auto", "segments", "exact"], default="auto",
                    help="radix joins: segment mode (no histogram pass) by size, always, or never")
    ap.add_argument("--wide", action="store_true",
                    help="radix joins: 16-byte tuples in every partition pass (HJ_F_WIDE), no 8-byte words")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-log", type=int, default=0,
                    help="log2 |R| of the CPU-baseline sample (0: pick by host memory)")
    return ap.parse_args()


def workload_config(a, n_gpus):
    return {
        "workload": f"{a.algo} PK-FK uniform, R=2^{a.nr_log} S=2^{a.ns_log} tuples of 16 B "
                    f"(int64 key + int64 row_id), {a.bits} radix bits, {a.passes} passes",
        "algo": a.algo,
        "r_tuples": 1 << a.nr_log,
        "s_tuples": 1 << a.ns_log,
        "num_radix_bits": a.bits,
        "num_passes": a.passes,
        "parallelism": f"{n_gpus} independent joins, one per GPU" if n_gpus > 1 else "1 GPU",
        "l2": "inputs (R+S = %.1f GB) larger than L2 (126 MB); no flush between steps"
              % (((1 << a.nr_log) + (1 << a.ns_log)) * 16 / 1e9),
        "generator": "seeded Feistel permutation (gen_pkfk_uniform distribution; the GPU arm generates it on "
                     "the device, the CPU baseline writes the same bytes to its .bin files)",
    }


# ---------------------------------------------------------------------------------------------
# GPU clock sampling during the timed region
# ---------------------------------------------------------------------------------------------
class ClockSampler:
    """SM clock, its maximum, power and the clock-event (throttle) reasons of this GPU, sampled every 5 ms
    through NVML in a background thread (nvidia-smi every 200 ms when NVML is not importable). stop()
    reports the samples inside the timed region when one is given (the host's bracket around the timed
    steps, which end with a synchronize), else those under load."""
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    BITS = (0x8, 0x40, 0x20, 0x4)  # NVML clock-event reason bits, in the order of NAMES
    FIELDS = ("index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, bus_id: str | None):
        self.bus_id = (bus_id or "").lower()
        self.samples = []  # (t, sm_mhz, max_mhz, reason_names, util)
        self.proc = None
        self.nvml = None
        self.stop_flag = threading.Event()

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        for i in range(pynvml.nvmlDeviceGetCount()):
            h = pynvml.nvmlDeviceGetHandleByIndex(i)
            bus = pynvml.nvmlDeviceGetPciInfo(h).busId
            bus = (bus.decode() if isinstance(bus, bytes) else bus).lower()
            if not self.bus_id or bus.endswith(self.bus_id):
                return pynvml, h
        return None

    def start(self):
        try:
            got = self._nvml_handle()
        except Exception:
            got = None
        if got:
            self.nvml, self.handle = got
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _poll(self):
        nv, h = self.nvml, self.handle
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop_flag.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                bits = get_reasons(h)
                util = nv.nvmlDeviceGetUtilizationRates(h).gpu
                names = [n for n, b in zip(self.NAMES, self.BITS) if bits & b]
                self.samples.append((time.monotonic(), float(sm), float(mx), names, float(util)))
            except Exception:
                pass
            time.sleep(0.005)

    def _read(self):
        def num(x):
            try:
                return float(x.split()[0])
            except (ValueError, IndexError):
                return None

        for line in self.proc.stdout:
            parts = [p.strip() for p in line.strip().split(",")]
            if len(parts) < 11 or (self.bus_id and not parts[1].lower().endswith(self.bus_id)):
                continue
            names = [n for i, n in enumerate(self.NAMES) if parts[6 + i].lower().startswith("active")]
            self.samples.append((time.monotonic(), num(parts[2]), num(parts[3]), names, num(parts[10]) or 0.0))

    def stop(self, window=None):
        if self.nvml:
            self.stop_flag.set()
            self.thread.join(timeout=2)
        elif self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)
        else:
            return None
        rows = [r for r in self.samples if r[1] is not None]
        if not rows:
            return None
        inside = [r for r in rows if window and window[0] <= r[0] <= window[1]]
        loaded = [r for r in rows if r[4] >= 50]
        use = inside or loaded or rows
        reasons = sorted({n for r in use for n in r[3]})
        return {"sm_mhz": statistics.median(r[1] for r in use), "sm_max_mhz": max(r[2] for r in rows),
                "reasons": reasons, "samples": len(rows), "samples_in_timed_region": len(inside),
                "samples_under_load": len(loaded), "source": "nvml" if self.nvml else "nvidia-smi"}


def reduce_over_ranks(value: float, dist, device, op: str = "max") -> float:
    """The max (or min) of a per-rank number over all ranks; the number itself without a process group.
    Every rank must call it at the same point (it is a collective)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.MIN)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, seconds: float) -> float:
    """Weak scaling: every rank processed units_per_rank; seconds is the slowest rank's time."""
    return world * units_per_rank / seconds


_MODE_SAMPLER = None  # clock sampler running over a whole non-headline mode (started in main)


def emit(rank: int, line: dict) -> None:
    """Rank 0 prints the one JSON line of the run (with the mode's clock record, when one is sampled)."""
    if _MODE_SAMPLER is not None and "clocks" not in line:
        line["clocks"] = _MODE_SAMPLER.stop()
    if rank == 0:
        print(json.dumps(line), flush=True)


def device_bus_id(torch, dev):
    try:
        pr = torch.cuda.get_device_properties(dev)
        return "%02x:%02x.0" % (int(pr.pci_bus_id), int(pr.pci_device_id))
    except (AttributeError, TypeError, ValueError):
        return None


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def traffic_profile(kernel: str):
    """Per-tuple DRAM traffic of a kernel from a committed ncu summary (profiles/<kernel>.json)."""
    p = ROOT / "profiles" / f"{kernel}.json"
    if not p.exists():
        return None
    return json.loads(p.read_text())


# ---------------------------------------------------------------------------------------------
# CPU baseline: the reference's own multithreaded join (oracle/_ref) on the host cores
# ---------------------------------------------------------------------------------------------
def host_mem_available_gb() -> float:
    try:
        for ln in open("/proc/meminfo"):
            if ln.startswith("MemAvailable:"):
                return int(ln.split()[1]) / 1e6
    except OSError:
        pass
    return 0.0


def cpu_reference_run(a, trials: int, warmup: int = 1, sample_log: int = 0):
    """The reference's own multithreaded join (oracle/_ref) on the host cores, on relations written by
    the oracle's restatement of the library's generator (the same bytes as the GPU arm's relations, made
    without loading the library). Runs warmup + trials trials and drops the first `warmup` (the
    reference drops one, src/main.c:434). Returns (throughput tuples/s per timed trial, sample
    description, threads, kind)."""
    orc = load_module("hj_oracle", ROOT / "oracle" / "hj_oracle.py")
    nr_log, ns_log = a.nr_log, a.ns_log
    if sample_log:
        ns_log = sample_log + (a.ns_log - a.nr_log)
        nr_log = sample_log
    else:
        # R+S files, the reference's private copy and its partition buffers: 3 x 16 B per tuple.
        need_gb = 3 * 16 * ((1 << nr_log) + (1 << ns_log)) / 1e9 + 4
        while host_mem_available_gb() < need_gb and nr_log > 20:
            nr_log -= 1
            ns_log -= 1
            need_gb /= 2
    nR, nS = 1 << nr_log, 1 << ns_log
    threads = os.cpu_count() or 1
    passes = a.passes
    if not orc.ref_available(passes):
        raise RuntimeError("oracle/_ref is not built")
    tmpdir = "/dev/shm" if os.path.isdir("/dev/shm") else None
    warmup = max(1, warmup)
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        orc.gen_fast_files(d, "r.bin", "s.bin", nR, nS, seed=12345, threads=threads)
        runs = orc.ref_run_files(a.algo.replace("_bw_reg", ""), d, "r.bin", "s.bin", nR, nS, bits=a.bits,
                                 passes=passes, threads=threads, trials=trials + warmup, timeout=1800)
    want = orc.pkfk_closed_form(nR, nS)
    for r in runs:
        if (r[0], r[1]) != want:
            raise RuntimeError(f"reference result {r[:2]} != closed form {want}")
    timed = runs[warmup:]
    thr = [(nR + nS) / r[4] for r in timed]
    sample = (f"{a.algo} R=2^{nr_log} S=2^{ns_log}, {len(timed)} timed trials after {warmup} warm-up, "
              "reference timekeeper total (buildpart + probejoin, src/algo/phj.c:2509-2511)")
    return thr, sample, threads, "reference"


# ---------------------------------------------------------------------------------------------
def run_reference_arm(a, rank, world):
    if rank != 0:
        return 0
    thr, sample, threads, kind = cpu_reference_run(a, trials=max(a.steps, 1), warmup=a.warmup,
                                                   sample_log=a.cpu_sample_log)
    value = statistics.mean(thr)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": len(thr),
        "warmup": max(1, a.warmup), "ms_per_step": ((1 << a.nr_log) + (1 << a.ns_log)) / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic", "config": workload_config(a, a.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(a, rank, world, local_rank):
    import torch

    hj = load_module("hashjoin_scm_b200", PKG_DIR / "__init__.py")
    hj.lib()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        dist = dist_mod
    nR, nS = 1 << a.nr_log, 1 << a.ns_log
    stream = torch.cuda.current_stream(dev)
    R = torch.empty((nR, 2), dtype=torch.int64, device=dev)
    S = torch.empty((nS, 2), dtype=torch.int64, device=dev)
    hj.gen_fast_device(nR, nS, R.data_ptr(), S.data_ptr(), seed=12345 + rank, stream=stream.cuda_stream)
    torch.cuda.synchronize(dev)
    want = hj.pkfk_closed_form(nR, nS)
    ctx = hj.Context(local_rank)
    pipe_flag = {"auto": 0, "segments": hj.HJ_F_SEGMENTS, "exact": hj.HJ_F_EXACT}[a.pipeline] | (
        hj.HJ_F_WIDE if a.wide else 0)
    # Timed steps carry no timing events (the library's own event records and elapsed-time queries
    # would add host work to every step); the phase breakdown comes from extra untimed steps.
    flags = hj.HJ_F_NO_TIMING | pipe_flag

    def step(fl=flags):
        r = hj.join(a.algo, R, S, on_device=True, bits=a.bits, passes=a.passes, device=local_rank,
                    stream=stream.cuda_stream, flags=fl, ctx=ctx)
        if (r.matched_cnt, r.checksum) != want:
            raise RuntimeError(f"wrong result {(r.matched_cnt, r.checksum)} != {want}")
        return r

    for _ in range(a.warmup):
        step()
    sampler = ClockSampler(device_bus_id(torch, dev))
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    sampler.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t_win0 = time.monotonic()
    e0.record(stream)
    results = [step() for _ in range(a.steps)]
    e1.record(stream)
    torch.cuda.synchronize(dev)
    t_win1 = time.monotonic()
    clocks = sampler.stop((t_win0, t_win1))
    if dist:
        dist.barrier()
    ms = reduce_over_ranks(e0.elapsed_time(e1), dist, dev)
    value = whole_job_rate((nR + nS) * a.steps, world, ms / 1e3)
    phase_runs = [step(hj.HJ_F_PHASE_TIMES | pipe_flag) for _ in range(3)]
    phases = {name: statistics.mean(r.phase[i] for r in phase_runs) for i, name in enumerate(hj.PHASES)}
    launches = sum(r.kernel_launches for r in results)
    seg_mode = a.algo.startswith("phj") and phases["hist"] == 0.0

    # Roofline of the dominant kernel. Radix joins: a partition pass reads and writes every tuple once
    # (32 B); when the last pass stores compact final partitions (8-byte words, HJ_RES_COMPACT_PARTITIONS)
    # it writes 8 B per tuple (24 B) and the join reads 8 B per tuple instead of 16. The pipeline with P
    # passes moves 16 (2P + 1) B per tuple, 64 B with compact final partitions at P = 2.
    # Non-partitioned joins: build and probe read every tuple and touch one 16-byte slot each (32 B).
    peak, peak_kind = measured_peaks()
    step_s = ms / 1e3 / a.steps
    compact = bool(results[-1].flags & hj.HJ_RES_COMPACT_PARTITIONS)
    words1 = bool(results[-1].flags & hj.HJ_RES_WORD_PASS1)
    ordered = bool(results[-1].flags & hj.HJ_RES_ORDERED_PASSES)
    if a.algo.startswith("phj"):
        P = results[-1].physical_passes
        # bytes per tuple of each pass: read + write; 8-byte words halve what a pass writes (and what the
        # next pass reads)
        if P == 2:
            pass_b = [16 + (8 if words1 else 16), (8 if words1 else 16) + (8 if compact else 16)]
        else:
            pass_b = [16 + (8 if compact else 16)]
        pass_t = [phases["pass1"], phases["pass2"]] if P == 2 else [phases["pass1"]]
        scatter_bytes = sum(pass_b) / len(pass_b) * (nR + nS)  # per launch, averaged like the times
        pass_s = statistics.mean(pass_t)
        achieved = scatter_bytes / pass_s / 1e9
        prof = traffic_profile("scatter_kernel")
        traffic = prof["dram_bytes_per_tuple"] * (nR + nS) if prof else None
        if seg_mode and words1:
            # ncu traffic of the two passes with 8-byte words (profiles/segment_passes_words.json), per
            # launch, averaged over the two passes like `achieved`
            pw = traffic_profile("segment_passes_words")
            traffic = ((pw["dram_bytes_per_tuple_pass1"] + pw["dram_bytes_per_tuple_pass2"]) / 2 * (nR + nS)
                       if pw else None)
        elif seg_mode:
            # per launch, averaged over the two passes like `achieved`
            p1 = traffic_profile("seg_pass1_kernel")
            key2 = "dram_bytes_per_tuple_pass2_compact" if compact else "dram_bytes_per_tuple_pass2"
            traffic = ((p1["dram_bytes_per_tuple"] + prof[key2]) / 2 * (nR + nS)
                       if p1 and prof and key2 in prof else None)
        kname = ("seg_pass1_kernel / scatter_kernel (mean of the two radix partition passes)" if seg_mode
                 else "scatter_kernel (radix partition passes, mean per launch)")
        roofline = {"kernel": kname, "bound": "hbm",
                    "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "peak_source": peak_kind, "traffic": traffic,
                    "algorithmic_bytes_per_launch": scatter_bytes, "launch_ms": pass_s * 1e3,
                    "per_pass": [{"bytes_per_tuple": b, "ms": t * 1e3, "gbs": b * (nR + nS) / t / 1e9,
                                  "frac": b * (nR + nS) / t / 1e9 / peak} for b, t in zip(pass_b, pass_t)]}
        per_tuple = sum(pass_b) + (8 if compact else 16)
        # the same time against the 16-byte-tuple model of the survey (32 B per pass, 16 B for the join)
        roofline["frac_of_tuple_model"] = (16 * (2 * P + 1) * (nR + nS) / step_s / 1e9) / peak
    else:
        per_tuple = 32
        join_bytes = per_tuple * (nR + nS)
        achieved = join_bytes / step_s / 1e9
        roofline = {"kernel": "non-partitioned build + probe (the whole join)", "bound": "hbm",
                    "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "peak_source": peak_kind, "traffic": None,
                    "algorithmic_bytes_per_launch": join_bytes, "launch_ms": step_s * 1e3}
    pipe_bytes = per_tuple * (nR + nS)
    pipeline = {"algorithmic_bytes_per_tuple": per_tuple, "bytes_per_step": pipe_bytes,
                "compact_final_partitions": compact, "word_pass1": words1 if a.algo.startswith("phj") else False,
                "ordered_passes": ordered,
                "achieved_gbs": pipe_bytes / step_s / 1e9, "frac": pipe_bytes / step_s / 1e9 / peak,
                "phase_ms": {k: v * 1e3 for k, v in phases.items()}}

    # End to end through the public C ABI with pinned host relations: copy in, join, read result.
    e2e = None
    if not a.no_e2e:
        Rh = torch.empty((nR, 2), dtype=torch.int64, pin_memory=True)
        Sh = torch.empty((nS, 2), dtype=torch.int64, pin_memory=True)
        Rh.copy_(R)
        Sh.copy_(S)
        del R, S
        torch.cuda.empty_cache()
        host_ctx = hj.Context(local_rank)

        def e2e_step():
            r = hj.join(a.algo, (Rh.data_ptr(), nR), (Sh.data_ptr(), nS), bits=a.bits, passes=a.passes,
                        device=local_rank, flags=hj.HJ_F_PINNED_HOST | pipe_flag, ctx=host_ctx)
            if (r.matched_cnt, r.checksum) != want:
                raise RuntimeError("wrong e2e result")
            return r

        e2e_step()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(a.e2e_steps):
            e2e_step()
        el = reduce_over_ranks(time.perf_counter() - t0, dist, dev)
        e2e = {"value": whole_job_rate((nR + nS) * a.e2e_steps, world, el), "unit": UNIT,
               "h2d_bytes_per_step": (nR + nS) * 16, "d2h_bytes_per_step": 64,
               "steps": a.e2e_steps, "ms_per_step": el / a.e2e_steps * 1e3}
        host_ctx.close()
        del Rh, Sh

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            thr, sample, threads, kind = cpu_reference_run(a, trials=2, sample_log=a.cpu_sample_log)
            cpu = {"value": statistics.mean(thr), "unit": UNIT, "cores": threads, "kind": kind, "sample": sample}
        except Exception as exc:  # the baseline is reported, not required
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {exc}"}
    ctx.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": workload_config(a, world),
            "partition_pipeline": (("segment mode: pass 1 writes segment chains and counts the histograms "
                                    "(no histogram pass)" if seg_mode else
                                    "exact offsets: histogram pass, then two scatter passes")
                                   if a.algo.startswith("phj") else None),
            "roofline": roofline, "pipeline": pipeline, "e2e": e2e, "cpu_baseline": cpu,
            "clocks": clocks, "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    return 0


def batch_workload(hj, torch, dev, njobs, seed=12345):
    """512 PK-FK joins: |R| log-uniform in [2^10, 2^22] (rounded up to a multiple of 256), |S| = k|R| with
    k uniform in 1..16, keys a seeded permutation per join (seed 12345 + i), uniform FKs."""
    import numpy as np

    rng = np.random.default_rng(seed)
    sizes = []
    for i in range(njobs):
        nR = int(2 ** rng.uniform(10, 22))
        nR = (nR + 255) // 256 * 256
        k = int(rng.integers(1, 17))
        sizes.append((nR, k * nR, k))
    total = sum(r + s for r, s, _ in sizes)
    buf = torch.empty((total, 2), dtype=torch.int64, device=dev)
    jobs, want, off = [], [], 0
    for i, (nR, nS, k) in enumerate(sizes):
        R = buf[off:off + nR]
        S = buf[off + nR:off + nR + nS]
        off += nR + nS
        hj.gen_fast_device(nR, nS, R.data_ptr(), S.data_ptr(), seed=seed + i)
        jobs.append(("phj_radix_bc", R, S))
        want.append(hj.pkfk_closed_form(nR, nS))
    torch.cuda.synchronize(dev)
    return jobs, want, total, buf


def run_batch_mode(a, rank, world, local_rank):
    import torch

    hj = load_module("hashjoin_scm_b200", PKG_DIR / "__init__.py")
    hj.lib()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    jobs, want, total, buf = batch_workload(hj, torch, dev, a.batch_jobs, seed=12345 + 1000 * rank)
    ctx = hj.Context(local_rank)
    # With --calibrate the batch is planned under several table budgets, each timed on the device; the
    # fastest plan is kept and its budget stays in the tuner (the tuned loop below uses it too).
    batch = hj.Batch(ctx, jobs, tune=a.calibrate)
    tuner = hj.tuner_get(ctx)
    calib = None

    def check(results):
        for r, w in zip(results, want):
            if (r.matched_cnt, r.checksum) != w:
                raise RuntimeError("batched join result differs from the closed form")

    # 1. plain per-join loop: every join through hj_join with the default algorithm and radix settings
    def loop(decided):
        out = []
        for algo, R, S in jobs:
            kw = {}
            if decided:
                import ctypes
                impl, bits, passes = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
                hj._bind_batch().hj_tuner_decide(ctx.handle, R.shape[0], S.shape[0], ctypes.byref(impl),
                                                 ctypes.byref(bits), ctypes.byref(passes))
                if impl.value == 0:
                    algo = "nphj_sc"
                else:
                    kw = {"bits": bits.value, "passes": passes.value}
            out.append(hj.join(algo, R, S, on_device=True, device=local_rank, ctx=ctx, flags=hj.HJ_F_NO_TIMING, **kw))
        return out

    def timed(fn, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(reps):
            res = fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / 1e3 / reps, res

    check(loop(False))
    t_loop, res = timed(lambda: loop(False), max(1, a.steps // 5))
    check(res)
    check(loop(True))
    t_loop_tuned, res = timed(lambda: loop(True), max(1, a.steps // 5))
    check(res)
    with batch as b:
        for _ in range(a.warmup):
            res, st = b.run()
            check(res)
        t_batch, (res, st) = timed(b.run, a.steps)
        check(res)
    n = len(jobs)
    dist = None
    if world > 1:
        import torch.distributed as dist
    t_loop = reduce_over_ranks(t_loop, dist, dev)
    t_loop_tuned = reduce_over_ranks(t_loop_tuned, dist, dev)
    t_batch = reduce_over_ranks(t_batch, dist, dev)
    if rank == 0:
        line = {
            "metric": "batched joins/s", "value": whole_job_rate(n, world, t_batch), "unit": "joins/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": t_batch * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": f"{n} PK-FK joins, |R| log-uniform in [2^10, 2^22] (multiple of 256), "
                                   "|S| = k|R|, k uniform in 1..16, 16-B tuples", "tuples": total},
            "per_join_loop": {"joins_per_s": n / t_loop, "ms": t_loop * 1e3, "algo": "phj_radix_bc, 14 bits, 2 passes"},
            "per_join_loop_tuned": {"joins_per_s": n / t_loop_tuned, "ms": t_loop_tuned * 1e3},
            "speedup_vs_loop": t_loop / t_batch, "speedup_vs_tuned_loop": t_loop_tuned / t_batch,
            "tuples_per_s": total / t_batch, "batch_stats": {"nphj_jobs": st.nphj_jobs, "phj_jobs": st.phj_jobs,
                                                             "waves": st.waves, "kernels": st.kernel_launches},
            "tuner": {"nphj_max_table_bytes": tuner.nphj_max_table_bytes, "calibrated": tuner.calibrated,
                      "phj_fixed_s": tuner.phj_fixed, "calibration": calib},
        }
    if rank == 0:
        emit(rank, line)
    ctx.close()
    return 0


def serve_workload(hj, torch, dev, n_small, seed):
    """Device-resident relations for served requests: n_small PK-FK pairs sized like the batched joins
    (|R| log-uniform in [2^10, 2^22], multiple of 256; |S| = k|R|, k uniform in 1..16) and one large pair
    of 2^26 x 2^28; every pair generated on the device with its own seed."""
    import numpy as np

    rng = np.random.default_rng(seed)
    sizes = []
    for i in range(n_small):
        nR = (int(2 ** rng.uniform(10, 22)) + 255) // 256 * 256
        k = int(rng.integers(1, 17))
        sizes.append((nR, k * nR))
    sizes.append((1 << 26, 1 << 28))
    total = sum(r + s for r, s in sizes)
    buf = torch.empty((total, 2), dtype=torch.int64, device=dev)
    pairs, off = [], 0
    for i, (nR, nS) in enumerate(sizes):
        R = buf[off:off + nR]
        S = buf[off + nR:off + nR + nS]
        off += nR + nS
        hj.gen_fast_device(nR, nS, R.data_ptr(), S.data_ptr(), seed=seed + i)
        pairs.append((R, S, hj.pkfk_closed_form(nR, nS)))
    torch.cuda.synchronize(dev)
    return pairs[:-1], pairs[-1], buf


def run_serve_mode(a, rank, world, local_rank):
    """Served joins: 95% of requests sized as the batched joins, 5% 2^26 x 2^28, relations device-resident.
    (1) Saturation: the whole request sequence submitted at once to the join server (continuous batching:
    small requests coalesced into waves, large ones on slots), against the plain per-join loop
    (phj_radix_bc, 14 bits, 2 passes for every request, as a caller of the reference's interface would
    run them) and the tuned loop (hj_join with the tuner's per-request decision), on the same sequence.
    (2) Latency: Poisson arrivals at each offered rate, server against the tuned loop."""
    import ctypes

    import numpy as np
    import torch

    hj = load_module("hashjoin_scm_b200", PKG_DIR / "__init__.py")
    hj.lib()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    small, big, buf = serve_workload(hj, torch, dev, 64, 12345 + 1000 * rank)
    rates = [float(x) for x in a.rates.split(",") if x]
    rng = np.random.default_rng(777 + rank)

    def picks_of(n):
        return [big if rng.random() < 0.05 else small[int(rng.integers(len(small)))] for _ in range(n)]

    sat_picks = picks_of(a.requests)
    streams = []
    for lam in rates:
        arrivals = np.cumsum(rng.exponential(1.0 / lam, a.requests))
        streams.append((lam, arrivals, picks_of(a.requests)))

    def pace(t_arr):
        while True:
            d = t_arr - hj.now()
            if d <= 0:
                return
            if d > 4e-4:
                time.sleep(d - 3e-4)

    def summarize(lat, picks, t0, t_last, n):
        lat = np.asarray(lat)
        small_lat = np.asarray([x for x, p in zip(lat, picks) if p is not big])
        return {"joins_per_s": n / (t_last - t0), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "max_ms": float(lat.max() * 1e3),
                "small_p50_ms": float(np.percentile(small_lat, 50) * 1e3),
                "small_p99_ms": float(np.percentile(small_lat, 99) * 1e3)}

    def check(c, want, what):
        if c.status or (c.matched_cnt, c.checksum) != want:
            raise RuntimeError(f"{what} result differs from the closed form")

    # 1. the join server: saturation, then the offered-rate sweep
    srv_out = []
    impl_counts = {0: 0, 1: 0}
    with hj.Server(local_rank, slots=a.slots, hbm_budget_bytes=a.budget_gb * 1e9, large_sm_share=a.large_share) as srv:
        for R, S, _ in small[:8] + [big]:  # warm-up: kernel attributes, first launches
            srv.wait_all([srv.submit("phj_radix_bc", R, S, on_device=True)])
        st0 = srv.stats()
        t0 = hj.now()
        ids = [srv.submit("phj_radix_bc", R, S, on_device=True) for R, S, _ in sat_picks]
        got = srv.wait_all(ids, timeout_s=600.0)
        t_last = max(c.done_s for c in got.values())
        for rid, (R, S, want) in zip(ids, sat_picks):
            check(got[rid], want, "served join")
        st1 = srv.stats()
        sat_server = {"joins_per_s": len(ids) / (t_last - t0), "seconds": t_last - t0,
                      "waves": st1.waves - st0.waves, "wave_requests": st1.wave_requests - st0.wave_requests,
                      "max_wave_size": max((c.wave_size for c in got.values()), default=0)}
        for lam, arrivals, picks in streams:
            t0 = hj.now() + 0.02
            ids = []
            for (R, S, _), t in zip(picks, arrivals):
                pace(t0 + t)
                ids.append(srv.submit("phj_radix_bc", R, S, on_device=True))
            got = srv.wait_all(ids, timeout_s=600.0)
            lat, t_last = [], t0
            for rid, (R, S, want), t in zip(ids, picks, arrivals):
                c = got[rid]
                check(c, want, "served join")
                lat.append(c.done_s - (t0 + t))
                t_last = max(t_last, c.done_s)
                impl_counts[c.impl] += 1
            srv_out.append(summarize(lat, picks, t0, t_last, len(ids)))
        st = srv.stats()
        peak, budget = st.peak_in_use_bytes, st.budget_bytes

    # 2. sequential per-join loops on the same sequences
    loop_out = []
    with hj.Context(local_rank) as ctx:
        # the same per-request decisions as the server's defaults (non-partitioned up to 16 MB tables)
        hj.tuner_set(ctx, nphj_max_table_bytes=16e6)

        def decided(R, S):
            impl, bits, passes = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            hj._bind_batch().hj_tuner_decide(ctx.handle, R.shape[0], S.shape[0], ctypes.byref(impl),
                                             ctypes.byref(bits), ctypes.byref(passes))
            return ("nphj_sc", {}) if impl.value == 0 else ("phj_radix_bc", {"bits": bits.value, "passes": passes.value})

        plans = {id(p[0]): decided(p[0], p[1]) for p in small + [big]}
        plain = ("phj_radix_bc", {"bits": 14, "passes": 2})

        def one(R, S, plan):
            algo, kw = plan
            return hj.join(algo, R, S, on_device=True, device=local_rank, ctx=ctx, flags=hj.HJ_F_NO_TIMING, **kw)

        for R, S, _ in small[:8] + [big]:
            one(R, S, plans[id(R)])
            one(R, S, plain)
        sat_loops = {}
        for name in ("plain", "tuned"):
            t_small = t_large = 0.0
            t0 = hj.now()
            for R, S, want in sat_picks:
                ta = hj.now()
                r = one(R, S, plain if name == "plain" else plans[id(R)])
                tb = hj.now()
                if (r.matched_cnt, r.checksum) != want:
                    raise RuntimeError(f"{name} loop result differs from the closed form")
                if R is big[0]:
                    t_large += tb - ta
                else:
                    t_small += tb - ta
            el = hj.now() - t0
            sat_loops[name] = {"joins_per_s": len(sat_picks) / el, "seconds": el, "large_requests_s": t_large,
                               "small_requests_s": t_small}
        for lam, arrivals, picks in streams:
            t0 = hj.now() + 0.02
            lat, t_last = [], t0
            for (R, S, want), t in zip(picks, arrivals):
                pace(t0 + t)
                r = one(R, S, plans[id(R)])
                done = hj.now()
                if (r.matched_cnt, r.checksum) != want:
                    raise RuntimeError("looped join result differs from the closed form")
                lat.append(done - (t0 + t))
                t_last = done
            loop_out.append(summarize(lat, picks, t0, t_last, len(picks)))

    # Amdahl: the server runs the large requests with the same partitioned pipeline as the plain loop, so
    # its speed-up over that loop is at most (the loop's total time) / (the loop's time on large requests).
    pl = sat_loops["plain"]
    bound = pl["seconds"] / pl["large_requests_s"] if pl["large_requests_s"] > 0 else None
    dist = None
    if world > 1:
        import torch.distributed as dist
    joins_s = world * reduce_over_ranks(sat_server["joins_per_s"], dist, dev, op="min")
    n_big = sum(1 for p in sat_picks if p is big)
    emit(rank, {
        "metric": "served joins/s at saturation (continuous batching), p50/p99 latency", "value": joins_s,
        "unit": "joins/s", "n_gpus": world, "steps": a.requests, "warmup": 9,
        "ms_per_step": 1e3 / sat_server["joins_per_s"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": "PK-FK join requests (phj_radix_bc semantics): 95% sized |R| log-uniform in "
                               "[2^10, 2^22], |S| = k|R| with k in 1..16, 5% 2^26 x 2^28; relations "
                               "device-resident", "requests": a.requests, "large_requests": n_big,
                   "slots": a.slots, "hbm_budget_bytes": budget, "peak_pool_bytes": peak},
        "saturation": {"server": sat_server, "plain_loop": sat_loops["plain"], "tuned_loop": sat_loops["tuned"],
                       "speedup_vs_plain_loop": sat_server["joins_per_s"] / sat_loops["plain"]["joins_per_s"],
                       "speedup_vs_tuned_loop": sat_server["joins_per_s"] / sat_loops["tuned"]["joins_per_s"],
                       "amdahl_bound_vs_plain_loop": bound},
        "sweep": [{"offered_rate": lam, "server": s_, "tuned_loop": l_}
                  for (lam, _, _), s_, l_ in zip(streams, srv_out, loop_out)],
        "impl_counts": {"nphj": impl_counts[0], "phj": impl_counts[1]},
    })
    del buf
    return 0


def dense_expected(torch, R, S, lp: bool):
    """Result of a join whose keys are dense in [0, K] computed by direct addressing on the device (an
    independent check, not the library): per key the build count, the wrapping sum of build row ids and
    the row id of the first build tuple in input order."""
    M = (1 << 64) - 1
    rk, rr = R[:, 0], R[:, 1]
    sk, sr = S[:, 0], S[:, 1]
    K = int(max(int(rk.max()), int(sk.max()))) + 1
    cnt = torch.bincount(rk, minlength=K)
    if lp:
        pos = torch.full((K,), R.shape[0], dtype=torch.int64, device=R.device)
        pos.scatter_reduce_(0, rk, torch.arange(R.shape[0], device=R.device), reduce="amin", include_self=True)
        hit = cnt[sk] > 0
        first = rr[pos.clamp(max=R.shape[0] - 1)]
        matched = int(hit.sum())
        checksum = int((torch.where(hit, first[sk] + sr, torch.zeros_like(sr))).sum()) & M
        return matched, checksum
    sumr = torch.zeros(K, dtype=torch.int64, device=R.device).index_add_(0, rk, rr)
    c = cnt[sk]
    matched = int(c.sum())
    checksum = int((sumr[sk] + c * sr).sum()) & M
    return matched, checksum


def run_skew_mode(a, rank, world, local_rank):
    """Config 3: R = 2^26 unique keys (a seeded permutation, row_id = key), S = 2^28 Zipf FK keys for
    theta in {0.5, 1.0, 1.5}; and the duplicate variant, R = 2^26 rows holding 2^24 distinct keys 4 times
    each, S = 2^28 uniform over those keys. phj_radix_lp (14 bits, 2 passes) and nphj_lp, inputs resident
    in HBM, every join checked against a direct-address count on the device."""
    import torch

    hj = load_module("hashjoin_scm_b200", PKG_DIR / "__init__.py")
    hj.lib()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream(dev)
    nR, nS = 1 << 26, 1 << 28
    R = torch.empty((nR, 2), dtype=torch.int64, device=dev)
    S = torch.empty((nS, 2), dtype=torch.int64, device=dev)
    ctx = hj.Context(local_rank)
    cases = []
    total_tuples, total_s = 0, 0.0
    data = [("zipf 0.5", 0.5, 1), ("zipf 1.0", 1.0, 1), ("zipf 1.5", 1.5, 1), ("dup x4", None, 4),
            ("build hot key", None, 0)]
    for name, theta, dup in data:
        seed = 12345 + 1000 * rank
        algos = ("phj_radix_lp", "nphj_lp")
        if name == "build hot key":
            # Build-side skew: a quarter of R (2^24 tuples) carries one key, so its radix partition holds
            # 2^24 build tuples; 1% of the probes carry that key (each matches 2^24 build tuples).
            # Non-partitioned tables cluster equal keys (quadratic build), so only the radix joins run.
            hj.gen_fast_device(nR, nS, R.data_ptr(), S.data_ptr(), seed=seed, stream=stream.cuda_stream)
            R[: nR // 4, 0] = 5
            S[::100, 0] = 5
            algos = ("phj_radix_bc", "phj_radix_lp")
        elif theta is None:
            hj.gen_fast_device(nR, nS, R.data_ptr(), S.data_ptr(), seed=seed, dup=dup, stream=stream.cuda_stream)
        else:
            hj.gen_fast_device(nR, 0, R.data_ptr(), S.data_ptr(), seed=seed, stream=stream.cuda_stream)
            hj.gen_zipf_device(nS, nR, theta, S.data_ptr(), seed=seed, stream=stream.cuda_stream)
        torch.cuda.synchronize(dev)
        for algo in algos:
            want = dense_expected(torch, R, S, lp=algo.endswith("_lp"))
            torch.cuda.synchronize(dev)

            def step():
                r = hj.join(algo, R, S, on_device=True, device=local_rank, stream=stream.cuda_stream,
                            flags=hj.HJ_F_PHASE_TIMES, ctx=ctx)
                if (r.matched_cnt, r.checksum) != want:
                    raise RuntimeError(f"{name} {algo}: {(r.matched_cnt, r.checksum)} != {want}")
                return r

            for _ in range(a.warmup):
                step()
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            res = [step() for _ in range(a.steps)]
            e1.record(stream)
            torch.cuda.synchronize(dev)
            sec = e0.elapsed_time(e1) / 1e3 / a.steps
            phases = {n: round(statistics.mean(r.phase[i] for r in res) * 1e3, 3) for i, n in enumerate(hj.PHASES)}
            cases.append({"data": name, "algo": algo, "ms": sec * 1e3, "tuples_per_s": (nR + nS) / sec,
                          "matched_cnt": want[0], "phase_ms": phases,
                          "large_partitions": int(res[-1].large_partitions)})
            total_tuples += nR + nS
            total_s += sec
    dist = None
    if world > 1:
        import torch.distributed as dist
    total_s = reduce_over_ranks(total_s, dist, dev)
    emit(rank, {
        "metric": "skew/duplicate lp joins (|R|+|S|)/s", "value": whole_job_rate(total_tuples, world, total_s),
        "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": total_s / len(cases) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": "R=2^26, S=2^28 16-B tuples: Zipf FK theta 0.5/1.0/1.5 over unique R keys, "
                               "R of 2^24 keys x4 with uniform S (phj_radix_lp, 14 bits / 2 passes, and nphj_lp); "
                               "and build-side skew: 2^24 of R's tuples on one key, 1% of probes on it "
                               "(phj_radix_bc and phj_radix_lp)",
                   "value": "all cases' tuples over all cases' time"},
        "cases": cases,
    })
    ctx.close()
    return 0


def run_mat_mode(a, rank, world, local_rank):
    """ptr_<algo> (default ptr_phj_radix_bc) on R = 2^nr, S = 2^ns PK-FK tuples whose row ids are
    1-based positions (the reference's payload data): every match written as an (r_row_id, s_row_id)
    pair into library scratch, then the retrieve phase gathers the checksum. Checked against the
    closed form |S|(|S|+1)/2 + m n(n+1)/2."""
    import torch

    hj = load_module("hashjoin_scm_b200", PKG_DIR / "__init__.py")
    hj.lib()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream(dev)
    nR, nS = 1 << a.nr_log, 1 << a.ns_log
    R = torch.empty((nR, 2), dtype=torch.int64, device=dev)
    S = torch.empty((nS, 2), dtype=torch.int64, device=dev)
    hj.gen_fast_device(nR, nS, R.data_ptr(), S.data_ptr(), seed=12345 + rank, payload=True, stream=stream.cuda_stream)
    torch.cuda.synchronize(dev)
    m = nS // nR
    want = (nS, (nS * (nS + 1) // 2 + m * nR * (nR + 1) // 2) % 2**64)
    ctx = hj.Context(local_rank)
    res = []
    for i in range(a.warmup + a.steps):
        r = hj.join_mat(a.algo, R, S, on_device=True, bits=a.bits, passes=a.passes, device=local_rank,
                        stream=stream.cuda_stream, ctx=ctx)
        if (r.matched_cnt, r.checksum) != want:
            raise RuntimeError(f"materialising join result {(r.matched_cnt, r.checksum)} != {want}")
        if i >= a.warmup:
            res.append(r)
    dist = None
    if world > 1:
        import torch.distributed as dist
    sec = reduce_over_ranks(statistics.mean(r.total for r in res), dist, dev)
    part = statistics.mean(r.buildpart for r in res)
    join = statistics.mean(r.probejoin for r in res)
    ret = statistics.mean(r.retrieve for r in res)
    hbm, src = measured_peaks()
    # Survey model: the 80 B/tuple pipeline plus 16 B written per pair; the retrieve phase reads each
    # pair (16 B) and gathers two row ids (a 32-B sector each).
    model = 80 * (nR + nS) + 16 * want[0]
    emit(rank, {
        "metric": "materialising join (|R|+|S|)/s", "value": whole_job_rate(nR + nS, world, sec), "unit": UNIT,
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": f"ptr_{a.algo} PK-FK, R=2^{a.nr_log} S=2^{a.ns_log}, row ids = positions, "
                               f"{a.bits} radix bits, {a.passes} passes; pairs in library scratch",
                   "pairs": want[0]},
        "phase_ms": {"partition": part * 1e3, "join_write_pairs": join * 1e3, "retrieve": ret * 1e3},
        "pipeline": {"model_bytes": model, "achieved_gbs": model / (part + join) / 1e9,
                     "frac_without_retrieve": model / (part + join) / 1e9 / hbm, "peak_gbs": hbm, "peak_source": src},
    })
    ctx.close()
    return 0


def run_stream_mode(a, rank, world, local_rank):
    """hj_join_streamed on PK-FK relations in pinned host memory: R = 2^28 tuples copied to the device
    once, S = 2^32 tuples (69 GB, more than the in-device pipeline can hold with R and its partition
    buffers) streamed through the device in chunks. Sizes shrink (halving S) when host memory is short.
    Reports the rate against the host-to-device link bound."""
    import torch

    hj = load_module("hashjoin_scm_b200", PKG_DIR / "__init__.py")
    L = hj.lib()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    nr_log, ns_log = 28, 32
    while ns_log > nr_log + 1 and host_mem_available_gb() < 1.3 * 16 * ((1 << nr_log) + (1 << ns_log)) / 1e9:
        ns_log -= 1
    nR, nS = 1 << nr_log, 1 << ns_log
    Rh = torch.empty((nR, 2), dtype=torch.int64, pin_memory=True)
    Sh = torch.empty((nS, 2), dtype=torch.int64, pin_memory=True)
    rc = L.hj_gen_fast_host(nR, nS, 12345 + rank, 0, 1, 0, Rh.data_ptr(), Sh.data_ptr())
    if rc:
        raise RuntimeError(f"hj_gen_fast_host failed: {rc}")
    want = hj.pkfk_closed_form(nR, nS)
    ctx = hj.Context(local_rank)
    res = []
    for i in range(a.warmup + a.steps):
        r = hj.join_streamed("phj_radix_bc", (Rh.data_ptr(), nR), (Sh.data_ptr(), nS), ctx, bits=14, passes=2)
        if (r.matched_cnt, r.checksum) != want:
            raise RuntimeError(f"streamed join result {(r.matched_cnt, r.checksum)} != {want}")
        if i >= a.warmup:
            res.append(r)
    dist = None
    if world > 1:
        import torch.distributed as dist
    sec = reduce_over_ranks(statistics.mean(r.total for r in res), dist, dev)
    link_s = (nR + nS) * 16 / 52e9  # measured pinned host-to-device copy rate of these machines
    emit(rank, {
        "metric": "streamed join (|R|+|S|)/s", "value": whole_job_rate(nR + nS, world, sec), "unit": UNIT,
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": f"phj_radix_bc PK-FK, R=2^{nr_log} on the device, S=2^{ns_log} streamed from pinned "
                               "host memory in chunks, 14 bits / 2 passes", "host_bytes": (nR + nS) * 16},
        "link_bound_ms": link_s * 1e3, "frac_of_link_bound": link_s / sec,
    })
    ctx.close()
    return 0


def main():
    a = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return run_reference_arm(a, rank, world)
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    if a.mode != "join":
        global _MODE_SAMPLER
        import torch

        _MODE_SAMPLER = ClockSampler(device_bus_id(torch, torch.device("cuda", local_rank)))
        _MODE_SAMPLER.start()
    try:
        if a.mode == "batch":
            return run_batch_mode(a, rank, world, local_rank)
        if a.mode == "serve":
            return run_serve_mode(a, rank, world, local_rank)
        if a.mode == "skew":
            return run_skew_mode(a, rank, world, local_rank)
        if a.mode == "mat":
            return run_mat_mode(a, rank, world, local_rank)
        if a.mode == "stream":
            return run_stream_mode(a, rank, world, local_rank)
        return run_ours(a, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
