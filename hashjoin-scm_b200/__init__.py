"""Python binding of libhjscm, the B200 equi-join hot path (C ABI in include/hjscm.h).

The library is the product; this module only loads it with ctypes and converts arguments. A join
takes two relations of 16-byte tuples {uint64 key, uint64 row_id} - numpy arrays of shape (n, 2) and
dtype uint64 on the host, or CUDA tensors / raw device pointers - and returns the reference's two
result values (match count, wrapping 64-bit checksum of r.row_id + s.row_id) with phase times.

The directory name contains a hyphen, so the package is loaded by path:
    spec = importlib.util.spec_from_file_location("hashjoin_scm_b200", ".../hashjoin-scm_b200/__init__.py")
"""
from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "lib" / "libhjscm.so"
MAIN_PATH = HERE / "bin" / "hj_main"

ALGOS = {
    "nphj_sc": 0,
    "nphj_lp": 1,
    "phj_radix_bc": 2,
    "phj_radix_lp": 3,
    # every match counted, as phj_radix_bc (src/algo/phj.c:683, 784, 881)
    "phj_radix_sc": 4,
    "phj_radix_hr": 5,
    "phj_radix_hro": 6,
}
# bandwidth-regulated aliases compute the same results (src/algo/phj_bw_reg.c:2874-2893); the
# asymmetric-radix names run with radix_bits_pass1 (src/algo/phj_asymm_radix.c)
for _s, _a in (("bc", 2), ("lp", 3), ("sc", 4), ("hr", 5), ("hro", 6)):
    ALGOS["phj_radix_bw_reg_" + _s] = _a
    if _s != "lp":
        ALGOS["phj_asymm_radix_" + _s] = _a
        ALGOS["phj_asymm_radix_bw_reg_" + _s] = _a
ASYMM_DEFAULT_BITS_PASS1 = 11

STATUS = {
    0: "HJ_OK",
    1: "HJ_E_INVAL",
    2: "HJ_E_OOM",
    3: "HJ_E_DEVICE",
    4: "HJ_E_PROBE_LIMIT",
    5: "HJ_E_TIMEOUT",
    6: "HJ_E_NOT_FOUND",
    7: "HJ_E_IO",
    8: "HJ_E_OVERFLOW",
    9: "HJ_E_BUDGET",
    10: "HJ_E_CAPACITY",
    11: "HJ_E_ROWID",
}
HJ_OK, HJ_E_INVAL, HJ_E_OOM, HJ_E_DEVICE, HJ_E_PROBE_LIMIT, HJ_E_TIMEOUT = 0, 1, 2, 3, 4, 5
HJ_E_NOT_FOUND, HJ_E_IO, HJ_E_OVERFLOW, HJ_E_BUDGET, HJ_E_CAPACITY, HJ_E_ROWID = 6, 7, 8, 9, 10, 11

HJ_F_NO_TIMING = 0x1
HJ_F_PINNED_HOST = 0x2
HJ_RES_COMPACT_PARTITIONS = 0x1
HJ_RES_WORD_PASS1 = 0x2
HJ_RES_ORDERED_PASSES = 0x4  # phj_radix_lp ran with ordered partition passes
HJ_F_PHASE_TIMES = 0x4
HJ_F_SEGMENTS = 0x20  # radix joins counting every match: segment mode at any size
HJ_F_EXACT = 0x40     # radix joins: always the histogram pass and exact pass-1 offsets
HJ_F_WIDE = 0x80      # radix joins: 16-byte tuples in every partition pass (no 8-byte words)
HJ_F_WORDS = 0x200    # radix joins: 8-byte words in every pass whenever the widths allow
HJ_F_ORDERED = 0x400  # phj_radix_lp: ordered partition passes at once (no unordered first run)
PHASES = ("hist", "plan", "pass1", "pass2", "join", "large")


class Params(ctypes.Structure):
    _fields_ = [
        ("num_radix_bits", ctypes.c_int),
        ("num_passes", ctypes.c_int),
        ("device", ctypes.c_int),
        ("inputs_on_device", ctypes.c_int),
        ("stream", ctypes.c_void_p),
        ("flags", ctypes.c_uint32),
        ("table_load", ctypes.c_double),
        ("radix_bits_pass1", ctypes.c_int),
        ("watchdog_ms", ctypes.c_int),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("matched_cnt", ctypes.c_uint64),
        ("checksum", ctypes.c_uint64),
        ("buildpart", ctypes.c_double),
        ("probejoin", ctypes.c_double),
        ("total", ctypes.c_double),
        ("h2d", ctypes.c_double),
        ("status", ctypes.c_int),
        ("physical_passes", ctypes.c_int),
        ("large_partitions", ctypes.c_uint64),
        ("phase", ctypes.c_double * 6),
        ("kernel_launches", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
        ("retrieve", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        d = {f: getattr(self, f) for f, _ in self._fields_ if f not in ("phase", "pad")}
        d["phase"] = list(self.phase)
        return d


class JoinError(RuntimeError):
    def __init__(self, status: int, what: str = "join"):
        super().__init__(f"{what} failed: {STATUS.get(status, status)}")
        self.status = status


_lib = None


def build(quiet: bool = True) -> None:
    """Compile libhjscm.so and hj_main in-tree (make, nvcc for sm_100a)."""
    out = subprocess.run(["make", "-C", str(HERE), "-j8"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("libhjscm build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])
    if not quiet:
        print(out.stdout)


def lib() -> ctypes.CDLL:
    """Load libhjscm.so (fails loudly when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run build() (make -C hashjoin-scm_b200)")
    L = ctypes.CDLL(str(LIB_PATH))
    u64, sz, vp, i32 = ctypes.c_uint64, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_int
    L.hj_params_init.argtypes = [ctypes.POINTER(Params)]
    L.hj_params_init.restype = None
    L.hj_status_str.argtypes = [i32]
    L.hj_status_str.restype = ctypes.c_char_p
    L.hj_algo_from_name.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
    L.hj_algo_from_name.restype = i32
    L.hj_algo_name.argtypes = [i32]
    L.hj_algo_name.restype = ctypes.c_char_p
    L.hj_ctx_create.argtypes = [i32, ctypes.POINTER(vp)]
    L.hj_ctx_create.restype = i32
    L.hj_ctx_destroy.argtypes = [vp]
    L.hj_ctx_destroy.restype = i32
    L.hj_ctx_reserve.argtypes = [vp, i32, ctypes.POINTER(Params), sz, sz]
    L.hj_ctx_reserve.restype = i32
    L.hj_ctx_scratch_bytes.argtypes = [vp]
    L.hj_ctx_scratch_bytes.restype = sz
    L.hj_join_ctx.argtypes = [vp, i32, ctypes.POINTER(Params), vp, sz, vp, sz, ctypes.POINTER(Result)]
    L.hj_join_ctx.restype = i32
    L.hj_join.argtypes = [i32, ctypes.POINTER(Params), vp, sz, vp, sz, ctypes.POINTER(Result)]
    L.hj_join.restype = i32
    L.hj_join_mat_ctx.argtypes = [vp, i32, ctypes.POINTER(Params), vp, sz, vp, sz, vp, sz, ctypes.POINTER(Result)]
    L.hj_join_mat_ctx.restype = i32
    L.hj_join_mat.argtypes = [i32, ctypes.POINTER(Params), vp, sz, vp, sz, vp, sz, ctypes.POINTER(Result)]
    L.hj_join_mat.restype = i32
    L.hj_join_streamed.argtypes = [vp, i32, ctypes.POINTER(Params), vp, sz, vp, sz, sz, ctypes.POINTER(Result)]
    L.hj_join_streamed.restype = i32
    L.hj_gen_pkfk_uniform.argtypes = [sz, sz, ctypes.c_uint, i32, vp, vp]
    L.hj_gen_pkfk_uniform.restype = i32
    L.hj_gen_dup_uniform.argtypes = [sz, sz, ctypes.c_uint, vp, vp]
    L.hj_gen_dup_uniform.restype = i32
    L.hj_gen_zipf.argtypes = [sz, sz, ctypes.c_double, ctypes.c_uint, vp]
    L.hj_gen_zipf.restype = i32
    L.hj_gen_fast_host.argtypes = [sz, sz, u64, i32, ctypes.c_uint, i32, vp, vp]
    L.hj_gen_fast_host.restype = i32
    L.hj_gen_fast_device.argtypes = [sz, sz, u64, i32, ctypes.c_uint, vp, vp, vp]
    L.hj_gen_fast_device.restype = i32
    L.hj_gen_zipf_device.argtypes = [sz, sz, ctypes.c_double, u64, vp, vp]
    L.hj_gen_zipf_device.restype = i32
    L.hj_pkfk_closed_form.argtypes = [sz, sz, ctypes.POINTER(u64), ctypes.POINTER(u64)]
    L.hj_pkfk_closed_form.restype = None
    L.hj_load_bin.argtypes = [ctypes.c_char_p, sz, vp]
    L.hj_load_bin.restype = i32
    L.hj_store_bin.argtypes = [ctypes.c_char_p, sz, vp]
    L.hj_store_bin.restype = i32
    _lib = L
    return L


def _ptr_len(rel, on_device: bool):
    """(pointer, tuple count) of a relation: numpy (n, 2) uint64, a CUDA tensor, or (ptr, n)."""
    if isinstance(rel, tuple):
        return int(rel[0]), int(rel[1])
    if on_device:
        # torch tensor of shape (n, 2) int64/uint64 on the GPU
        assert rel.is_cuda and rel.is_contiguous() and rel.element_size() == 8
        return int(rel.data_ptr()), int(rel.numel() // 2)
    arr = np.ascontiguousarray(rel)
    assert arr.dtype == np.uint64 and arr.ndim == 2 and arr.shape[1] == 2, "relations are (n, 2) uint64"
    return arr.ctypes.data, arr.shape[0]


def make_params(bits: int = 14, passes: int = 2, device: int = 0, on_device: bool = False,
                stream: int | None = None, flags: int = 0, load: float = 0.0, bits_pass1: int = 0,
                watchdog_ms: int = 0) -> Params:
    p = Params()
    lib().hj_params_init(ctypes.byref(p))
    p.num_radix_bits, p.num_passes, p.device = bits, passes, device
    p.inputs_on_device = 1 if on_device else 0
    p.stream = stream or None
    p.flags = flags
    p.table_load = load
    p.radix_bits_pass1 = bits_pass1
    p.watchdog_ms = watchdog_ms
    return p


def join(algo: str, R, S, *, bits: int = 14, passes: int = 2, device: int = 0, on_device: bool = False,
         stream: int | None = None, flags: int = 0, load: float = 0.0, ctx: "Context | None" = None,
         check: bool = True, bits_pass1: int | None = None, watchdog_ms: int = 0) -> Result:
    """Run one join (synchronous). Raises JoinError on a non-zero status when check is set.
    bits_pass1: pass-1 radix bits of a two-pass join (None: 11 for phj_asymm_radix_* names, as the
    reference's NUM_RADIX_BITS_PASS1 default, else an even split). load: the non-partitioned joins'
    table load factor (0: 0.4 for build relations up to 5 M tuples, 0.5 above)."""
    L = lib()
    a = ALGOS[algo]
    if bits_pass1 is None:
        bits_pass1 = ASYMM_DEFAULT_BITS_PASS1 if algo.startswith("phj_asymm_radix") else 0
    p = make_params(bits, passes, device, on_device, stream, flags, load, bits_pass1, watchdog_ms)
    pr, nr = _ptr_len(R, on_device)
    ps, ns = _ptr_len(S, on_device)
    res = Result()
    if ctx is not None:
        rc = L.hj_join_ctx(ctx.handle, a, ctypes.byref(p), pr, nr, ps, ns, ctypes.byref(res))
    else:
        rc = L.hj_join(a, ctypes.byref(p), pr, nr, ps, ns, ctypes.byref(res))
    if check and rc != 0:
        raise JoinError(rc, algo)
    res.status = rc
    return res


def join_mat(algo: str, R, S, *, pairs=None, pair_cap: int | None = None, bits: int = 14, passes: int = 2,
             device: int = 0, on_device: bool = False, stream: int | None = None, flags: int = 0,
             load: float = 0.0, ctx: "Context | None" = None, check: bool = True,
             bits_pass1: int | None = None) -> Result:
    """Materialising join (the reference's ptr_* joins; a "ptr_" prefix on algo is accepted): one
    (r.row_id, s.row_id) pair per match, checksum recomputed by the retrieve phase. pairs: None (kept
    in library scratch), a CUDA tensor (n, 2) int64 when on_device, or a numpy (n, 2) uint64 array."""
    L = lib()
    name = algo[4:] if algo.startswith("ptr_") else algo
    a = ALGOS[name]
    if bits_pass1 is None:
        bits_pass1 = ASYMM_DEFAULT_BITS_PASS1 if name.startswith("phj_asymm_radix") else 0
    p = make_params(bits, passes, device, on_device, stream, flags, load, bits_pass1)
    pr, nr = _ptr_len(R, on_device)
    ps, ns = _ptr_len(S, on_device)
    pp, cap = (None, 0)
    if pairs is not None:
        pp, cap = _ptr_len(pairs, on_device)
        if pair_cap is not None:
            cap = min(cap, pair_cap)
    res = Result()
    if ctx is not None:
        rc = L.hj_join_mat_ctx(ctx.handle, a, ctypes.byref(p), pr, nr, ps, ns, pp, cap, ctypes.byref(res))
    else:
        rc = L.hj_join_mat(a, ctypes.byref(p), pr, nr, ps, ns, pp, cap, ctypes.byref(res))
    if check and rc != 0:
        raise JoinError(rc, algo)
    res.status = rc
    return res


def join_streamed(algo: str, R, S, ctx: "Context", *, chunk_tuples: int = 0, bits: int = 14, passes: int = 2,
                  flags: int = 0, load: float = 0.0, check: bool = True, bits_pass1: int | None = None) -> Result:
    """Streamed join (hj_join_streamed): R stays on the device, S streams from host memory in chunks.
    R and S are host relations: numpy (n, 2) uint64 arrays or (pointer, n) pairs (pinned memory copies
    at full link speed)."""
    L = lib()
    a = ALGOS[algo]
    if bits_pass1 is None:
        bits_pass1 = ASYMM_DEFAULT_BITS_PASS1 if algo.startswith("phj_asymm_radix") else 0
    p = make_params(bits, passes, ctx.device, False, None, flags, load, bits_pass1)
    pr, nr = _ptr_len(R, False)
    ps, ns = _ptr_len(S, False)
    res = Result()
    rc = L.hj_join_streamed(ctx.handle, a, ctypes.byref(p), pr, nr, ps, ns, chunk_tuples, ctypes.byref(res))
    if check and rc != 0:
        raise JoinError(rc, algo)
    res.status = rc
    return res


class Context:
    """A library context: own stream, events and device scratch arena (hj_ctx_t)."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        rc = lib().hj_ctx_create(device, ctypes.byref(h))
        if rc:
            raise JoinError(rc, "hj_ctx_create")
        self.handle = h
        self.device = device

    def reserve(self, algo: str, nR: int, nS: int, **kw) -> None:
        p = make_params(device=self.device, **kw)
        rc = lib().hj_ctx_reserve(self.handle, ALGOS[algo], ctypes.byref(p), nR, nS)
        if rc:
            raise JoinError(rc, "hj_ctx_reserve")

    def scratch_bytes(self) -> int:
        return lib().hj_ctx_scratch_bytes(self.handle)

    def close(self) -> None:
        if self.handle:
            lib().hj_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def empty_relation(n: int) -> np.ndarray:
    return np.zeros((n, 2), dtype=np.uint64)


def gen_pkfk_uniform(nR: int, nS: int, seed: int = 12345, payload: bool = False):
    """Exact replay of the reference's gen_pkfk_uniform / payload_gen_pkfk_uniform (src/gen.c)."""
    R, S = empty_relation(nR), empty_relation(nS)
    rc = lib().hj_gen_pkfk_uniform(nR, nS, seed, 1 if payload else 0, R.ctypes.data, S.ctypes.data)
    if rc:
        raise JoinError(rc, "hj_gen_pkfk_uniform")
    return R, S


def gen_dup_uniform(nR: int, nS: int, seed: int = 12345):
    """Exact replay of the reference's gen_dup_uniform (src/gen.c:286-331)."""
    R, S = empty_relation(nR), empty_relation(nS)
    rc = lib().hj_gen_dup_uniform(nR, nS, seed, R.ctypes.data, S.ctypes.data)
    if rc:
        raise JoinError(rc, "hj_gen_dup_uniform")
    return R, S


def gen_zipf(nS: int, nR: int, factor: float, seed: int = 12345):
    """Exact replay of the reference's gen_zipf (src/inc/eth_genzipf.c:97-147) with the given factor."""
    S = empty_relation(nS)
    rc = lib().hj_gen_zipf(nS, nR, factor, seed, S.ctypes.data)
    if rc:
        raise JoinError(rc, "hj_gen_zipf")
    return S


def gen_fast_host(nR: int, nS: int, seed: int = 12345, payload: bool = False, dup: int = 1, threads: int = 0):
    R, S = empty_relation(nR), empty_relation(nS)
    rc = lib().hj_gen_fast_host(nR, nS, seed, 1 if payload else 0, dup, threads, R.ctypes.data, S.ctypes.data)
    if rc:
        raise JoinError(rc, "hj_gen_fast_host")
    return R, S


def gen_fast_device(nR: int, nS: int, R_ptr: int, S_ptr: int, seed: int = 12345, payload: bool = False,
                    dup: int = 1, stream: int | None = None) -> None:
    rc = lib().hj_gen_fast_device(nR, nS, seed, 1 if payload else 0, dup, R_ptr, S_ptr, stream or None)
    if rc:
        raise JoinError(rc, "hj_gen_fast_device")


def gen_zipf_device(nS: int, nR: int, factor: float, S_ptr: int, seed: int = 12345,
                    stream: int | None = None) -> None:
    rc = lib().hj_gen_zipf_device(nS, nR, factor, seed, S_ptr, stream or None)
    if rc:
        raise JoinError(rc, "hj_gen_zipf_device")


def pkfk_closed_form(nR: int, nS: int) -> tuple[int, int]:
    m, c = ctypes.c_uint64(), ctypes.c_uint64()
    lib().hj_pkfk_closed_form(nR, nS, ctypes.byref(m), ctypes.byref(c))
    return m.value, c.value


def header_functions() -> list[str]:
    """Names of every function declared in include/*.h (for export checks)."""
    import re

    names = []
    inc = HERE.parent / "include"
    for h in sorted(inc.glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([a-z_][a-z0-9_]*)\s*\([^;{]*\)\s*;", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof"):
                names.append(name)
    return sorted(set(names))


# ---------------------------------------------------------------------------------------------
# Batched joins and the autotuner (include/hjscm.h, "Batched joins")
# ---------------------------------------------------------------------------------------------
HJ_F_NO_GRAPH = 0x8
HJ_F_TUNE = 0x10
HJ_F_TEST_STALL = 0x100
IMPL_NAMES = {0: "nphj", 1: "phj"}


TUNER_LEVELS = 8


class Tuner(ctypes.Structure):
    _fields_ = [("nphj_max_table_bytes", ctypes.c_double), ("wave_table_bytes", ctypes.c_double),
                ("partition_target", ctypes.c_int), ("calibrated", ctypes.c_int),
                ("level_nR", ctypes.c_double * TUNER_LEVELS), ("nphj_build", ctypes.c_double * TUNER_LEVELS),
                ("nphj_probe", ctypes.c_double * TUNER_LEVELS), ("phj", ctypes.c_double * TUNER_LEVELS),
                ("phj_fixed", ctypes.c_double)]


class BatchJob(ctypes.Structure):
    _fields_ = [("algo", ctypes.c_int), ("R", ctypes.c_void_p), ("nR", ctypes.c_size_t), ("S", ctypes.c_void_p),
                ("nS", ctypes.c_size_t)]


class BatchResult(ctypes.Structure):
    _fields_ = [("matched_cnt", ctypes.c_uint64), ("checksum", ctypes.c_uint64), ("status", ctypes.c_int),
                ("impl", ctypes.c_int), ("num_radix_bits", ctypes.c_int), ("num_passes", ctypes.c_int)]


class BatchStats(ctypes.Structure):
    _fields_ = [("seconds", ctypes.c_double), ("kernel_launches", ctypes.c_uint32), ("waves", ctypes.c_int),
                ("nphj_jobs", ctypes.c_int), ("phj_jobs", ctypes.c_int)]


def _bind_batch():
    L = lib()
    if getattr(L, "_batch_bound", False):
        return L
    vp, i32, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
    L.hj_tuner_get.argtypes = [vp, ctypes.POINTER(Tuner)]
    L.hj_tuner_set.argtypes = [vp, ctypes.POINTER(Tuner)]
    L.hj_tuner_decide.argtypes = [vp, sz, sz, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i32)]
    L.hj_tuner_calibrate.argtypes = [vp, ctypes.POINTER(ctypes.c_double), i32]
    L.hj_batch_plan.argtypes = [vp, ctypes.POINTER(BatchJob), i32, ctypes.POINTER(Params), ctypes.POINTER(vp)]
    L.hj_batch_run.argtypes = [vp, ctypes.POINTER(BatchResult), ctypes.POINTER(BatchStats)]
    L.hj_batch_destroy.argtypes = [vp]
    for f in ("hj_tuner_get", "hj_tuner_set", "hj_tuner_decide", "hj_tuner_calibrate", "hj_batch_plan",
              "hj_batch_run", "hj_batch_destroy"):
        getattr(L, f).restype = i32
    L._batch_bound = True
    return L


def tuner_get(ctx: "Context") -> Tuner:
    t = Tuner()
    _bind_batch().hj_tuner_get(ctx.handle, ctypes.byref(t))
    return t


def tuner_set(ctx: "Context", **kw) -> Tuner:
    t = tuner_get(ctx)
    for k, v in kw.items():
        setattr(t, k, v)
    rc = _bind_batch().hj_tuner_set(ctx.handle, ctypes.byref(t))
    if rc:
        raise JoinError(rc, "hj_tuner_set")
    return t


def tuner_calibrate(ctx: "Context"):
    """Time both implementations on the device and set the crossover; returns [(|R|, t_nphj, t_phj)]."""
    rep = (ctypes.c_double * 24)()
    rc = _bind_batch().hj_tuner_calibrate(ctx.handle, rep, 24)
    if rc:
        raise JoinError(rc, "hj_tuner_calibrate")
    return [(int(rep[3 * i]), rep[3 * i + 1], rep[3 * i + 2]) for i in range(8) if rep[3 * i] > 0]


class Batch:
    """A planned batch of joins on device-resident relations (hj_batch_plan); run() launches it once.

    jobs: list of (algo name, R, S) where R and S are CUDA tensors of shape (n, 2) or (pointer, n)."""

    def __init__(self, ctx: "Context", jobs, graph: bool = True, tune: bool = False):
        L = _bind_batch()
        arr = (BatchJob * max(len(jobs), 1))()
        self._keep = []
        for i, (algo, R, S) in enumerate(jobs):
            pr, nr = _ptr_len(R, True)
            ps, ns = _ptr_len(S, True)
            arr[i].algo, arr[i].R, arr[i].nR, arr[i].S, arr[i].nS = ALGOS[algo], pr, nr, ps, ns
            self._keep.append((R, S))
        p = make_params(device=ctx.device, on_device=True,
                        flags=(0 if graph else HJ_F_NO_GRAPH) | (HJ_F_TUNE if tune else 0))
        h = ctypes.c_void_p()
        rc = L.hj_batch_plan(ctx.handle, arr, len(jobs), ctypes.byref(p), ctypes.byref(h))
        if rc:
            raise JoinError(rc, "hj_batch_plan")
        self.handle, self.n = h, len(jobs)

    def run(self):
        res = (BatchResult * max(self.n, 1))()
        st = BatchStats()
        rc = _bind_batch().hj_batch_run(self.handle, res, ctypes.byref(st))
        if rc:
            raise JoinError(rc, "hj_batch_run")
        return list(res)[: self.n], st

    def close(self):
        if self.handle:
            _bind_batch().hj_batch_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---------------------------------------------------------------------------------------------
# Join server (include/hjscm.h, "Join server")
# ---------------------------------------------------------------------------------------------
class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("slots", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_double),
                ("autotune", ctypes.c_int), ("tuner", Tuner), ("small_request_tuples", ctypes.c_double),
                ("large_sm_share", ctypes.c_double), ("waves", ctypes.c_int), ("wave_max_requests", ctypes.c_int),
                ("max_large_inflight", ctypes.c_int)]


class Completion(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("matched_cnt", ctypes.c_uint64), ("checksum", ctypes.c_uint64),
                ("status", ctypes.c_int), ("impl", ctypes.c_int), ("submit_s", ctypes.c_double),
                ("start_s", ctypes.c_double), ("done_s", ctypes.c_double), ("wave", ctypes.c_uint64),
                ("wave_size", ctypes.c_int), ("reserved", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("admitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("budget_bytes", ctypes.c_double), ("in_use_bytes", ctypes.c_double),
                ("peak_in_use_bytes", ctypes.c_double), ("queued", ctypes.c_int), ("inflight", ctypes.c_int),
                ("waves", ctypes.c_uint64), ("wave_requests", ctypes.c_uint64)]


def _bind_server():
    L = _bind_batch()
    if getattr(L, "_server_bound", False):
        return L
    vp, i32, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
    L.hj_now.argtypes = []
    L.hj_now.restype = ctypes.c_double
    L.hj_server_config_init.argtypes = [ctypes.POINTER(ServerConfig)]
    L.hj_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
    L.hj_server_submit.argtypes = [vp, i32, vp, sz, vp, sz, i32, ctypes.POINTER(ctypes.c_uint64)]
    L.hj_server_poll.argtypes = [vp, ctypes.POINTER(Completion), i32, ctypes.POINTER(i32), i32]
    L.hj_server_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
    L.hj_server_destroy.argtypes = [vp]
    for f in ("hj_server_config_init", "hj_server_create", "hj_server_submit", "hj_server_poll",
              "hj_server_stats", "hj_server_destroy"):
        getattr(L, f).restype = i32
    L._server_bound = True
    return L


def now() -> float:
    """The library's monotonic clock (seconds), the one server completions are stamped with."""
    return _bind_server().hj_now()


class Server:
    """A join server (hj_server_t): submit() queues a join and returns its id at once; poll() returns
    completions. Relations are numpy (n, 2) uint64 arrays (host) or CUDA tensors (on_device=True); the
    server keeps a reference to them until their completion has been polled."""

    def __init__(self, device: int = 0, slots: int = 8, hbm_budget_bytes: float = 150e9, autotune: bool = True,
                 tuner: dict | None = None, large_sm_share: float | None = None, waves: bool = True,
                 wave_max_requests: int | None = None, max_large_inflight: int | None = None):
        L = _bind_server()
        cfg = ServerConfig()
        L.hj_server_config_init(ctypes.byref(cfg))
        cfg.device, cfg.slots, cfg.hbm_budget_bytes, cfg.autotune = device, slots, hbm_budget_bytes, int(autotune)
        cfg.waves = int(waves)
        if wave_max_requests is not None:
            cfg.wave_max_requests = wave_max_requests
        if max_large_inflight is not None:
            cfg.max_large_inflight = max_large_inflight
        for k, v in (tuner or {}).items():
            setattr(cfg.tuner, k, v)
        if large_sm_share is not None:
            cfg.large_sm_share = large_sm_share
        h = ctypes.c_void_p()
        rc = L.hj_server_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc:
            raise JoinError(rc, "hj_server_create")
        self.handle = h
        self._keep = {}

    def submit(self, algo: str, R, S, on_device: bool = False) -> int:
        if not on_device:
            R = np.ascontiguousarray(R)
            S = np.ascontiguousarray(S)
        pr, nr = _ptr_len(R, on_device)
        ps, ns = _ptr_len(S, on_device)
        rid = ctypes.c_uint64()
        rc = _bind_server().hj_server_submit(self.handle, ALGOS[algo], pr, nr, ps, ns, int(on_device),
                                             ctypes.byref(rid))
        if rc:
            raise JoinError(rc, "hj_server_submit")
        self._keep[rid.value] = (R, S)
        return rid.value

    def poll(self, max_n: int = 256, wait_ms: int = 0) -> list:
        buf = (Completion * max_n)()
        n = ctypes.c_int()
        rc = _bind_server().hj_server_poll(self.handle, buf, max_n, ctypes.byref(n), wait_ms)
        if rc:
            raise JoinError(rc, "hj_server_poll")
        out = list(buf)[: n.value]
        for c in out:
            self._keep.pop(c.id, None)
        return out

    def wait_all(self, ids, timeout_s: float = 120.0) -> dict:
        """Poll until every id in ids has completed; returns {id: Completion}."""
        want, got = set(ids), {}
        t_end = now() + timeout_s
        while want - set(got):
            if now() > t_end:
                raise JoinError(HJ_E_TIMEOUT, "hj_server_poll")
            for c in self.poll(wait_ms=50):
                got[c.id] = c
        return got

    def stats(self) -> ServerStats:
        st = ServerStats()
        _bind_server().hj_server_stats(self.handle, ctypes.byref(st))
        return st

    def close(self):
        if self.handle:
            _bind_server().hj_server_destroy(self.handle)
            self.handle = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ------------------------------------------------------------------------------------------------
# Sharded joins: one join over the GPUs of a torch.distributed process group
# ------------------------------------------------------------------------------------------------
def shard_route(T, nshards: int, stream: int | None = None):
    """Group the tuples of a CUDA tensor T (n, 2) int64 by owner rank (hj_shard_route, stable: input
    order kept within each owner's range). Returns (routed tensor, counts) with counts an int64 CUDA
    tensor of nshards entries."""
    import torch

    L = lib()
    if not getattr(L, "_shard_bound", False):
        L.hj_shard_route_scratch_bytes.argtypes = [ctypes.c_size_t, ctypes.c_int]
        L.hj_shard_route_scratch_bytes.restype = ctypes.c_size_t
        L.hj_shard_route.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
        L.hj_shard_route.restype = ctypes.c_int
        L._shard_bound = True
    if not T.is_cuda:
        raise ValueError("shard_route takes a CUDA tensor")
    n = T.shape[0]
    out = torch.empty_like(T)
    counts = torch.empty(nshards, dtype=torch.int64, device=T.device)
    sb = L.hj_shard_route_scratch_bytes(n, nshards)
    scratch = torch.empty(sb, dtype=torch.uint8, device=T.device)
    st = stream if stream is not None else torch.cuda.current_stream(T.device).cuda_stream
    rc = L.hj_shard_route(T.data_ptr() if n else None, n, nshards, out.data_ptr() if n else None, counts.data_ptr(),
                          scratch.data_ptr(), sb, st)
    if rc:
        raise JoinError(rc, "hj_shard_route")
    return out, counts


def sharded_join(algo: str, R, S, *, group=None, bits: int = 14, passes: int = 2, ctx: "Context | None" = None,
                 route=None, local_join=None) -> tuple[int, int]:
    """One join of the relations spread over the ranks of a torch.distributed process group: rank r
    holds R_r and S_r (CUDA tensors (n, 2) int64), and the join is that of R = R_0 ++ R_1 ++ ... and
    S = S_0 ++ S_1 ++ ... (first-match joins take the first build tuple in that order). Every rank
    routes its tuples to their owner ranks (hj_shard_route), one all-to-all moves them (counts first),
    each rank joins what it owns on its GPU, and an all-reduce adds the (matched_cnt, check_sum) pairs
    modulo 2^64. Returns the same pair on every rank. Every rank must call it with the same arguments.

    route(T, nshards) -> (routed, counts) and local_join(algo, R, S) -> (matched, checksum) replace the
    GPU routing kernel and the GPU join (defaults); tests of the exchange on CPU-only process groups
    pass host implementations of both."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    if route is None:
        route = shard_route
    if local_join is None:
        def local_join(a, r, s):
            res = join(a, r, s, on_device=True, bits=bits, passes=passes, device=r.device.index or 0, ctx=ctx)
            return res.matched_cnt, res.checksum

    def exchange(T):
        routed, counts = route(T, world)
        counts = counts.to(torch.int64)
        recv_counts = torch.empty_like(counts)
        dist.all_to_all_single(recv_counts, counts, group=group)
        send, recv = counts.tolist(), recv_counts.tolist()
        out = torch.empty((sum(recv), 2), dtype=T.dtype, device=T.device)
        dist.all_to_all_single(out, routed, output_split_sizes=recv, input_split_sizes=send, group=group)
        return out

    Rx, Sx = exchange(R), exchange(S)
    matched, checksum = local_join(algo, Rx, Sx)

    def signed(x):
        x &= (1 << 64) - 1
        return x - (1 << 64) if x >= 1 << 63 else x

    t = torch.tensor([signed(matched), signed(checksum)], dtype=torch.int64, device=R.device)
    dist.all_reduce(t, group=group)  # two's-complement sums wrap exactly as the u64 sums do
    m, c = t.tolist()
    return m & ((1 << 64) - 1), c & ((1 << 64) - 1)
