"""The allocation-free join entry point (hj_nphj_join_noalloc), through the C ABI.

It exists for callers that cannot allocate device memory (an engine that owns the GPU's memory, or a
request loop that must not call the CUDA allocator): its table lives in a fixed array of the library.
Two calls in a row on different relations must each give the result of the regular entry point
(hj_join) and of the oracle, bit for bit: the second call must not see the first call's table contents.
Repeated calls must leave the device's free memory unchanged, and the largest build relation the
array holds must join correctly.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class DeviceResult(ctypes.Structure):
    _fields_ = [("matched_cnt", ctypes.c_uint64), ("checksum", ctypes.c_uint64), ("error_bits", ctypes.c_uint32),
                ("reserved0", ctypes.c_uint32), ("reserved", ctypes.c_uint64 * 5)]


def _bind(hj):
    L = hj.lib()
    f = L.hj_nphj_join_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _relations(seed, nR, nS, key_range):
    rng = np.random.default_rng(seed)
    R = np.empty((nR, 2), dtype=np.uint64)
    S = np.empty((nS, 2), dtype=np.uint64)
    R[:, 0] = rng.integers(1, key_range, nR, dtype=np.uint64)  # duplicates on the build side
    S[:, 0] = rng.integers(1, key_range + key_range // 4, nS, dtype=np.uint64)  # some probes miss
    R[:, 1] = rng.integers(0, 2**63, nR, dtype=np.uint64)
    S[:, 1] = rng.integers(0, 2**63, nS, dtype=np.uint64)
    return R, S


def test_noalloc_matches_regular_entry_point_twice(hj, oracle, cuda):
    noalloc = _bind(hj)
    datasets = [_relations(1, 200_000, 700_000, 150_000), _relations(2, 50_000, 300_000, 40_000)]
    out = cuda.zeros(8, dtype=cuda.int64, device="cuda")
    stream = cuda.cuda.current_stream()
    for algo in ("nphj_sc", "nphj_lp"):
        for R, S in datasets:  # two calls in a row through the shared array
            Rd = cuda.from_numpy(R.view(np.int64)).cuda()
            Sd = cuda.from_numpy(S.view(np.int64)).cuda()
            rc = noalloc(hj.ALGOS[algo], Rd.data_ptr(), R.shape[0], Sd.data_ptr(), S.shape[0], out.data_ptr(),
                         stream.cuda_stream)
            assert rc == 0
            stream.synchronize()
            got = DeviceResult.from_buffer_copy(out.cpu().numpy().tobytes())
            want = hj.join(algo, Rd, Sd, on_device=True)
            assert got.error_bits == 0
            assert (got.matched_cnt, got.checksum) == (want.matched_cnt, want.checksum), algo
            assert (got.matched_cnt, got.checksum) == oracle.join(algo, R, S), algo


def _call(noalloc, hj, cuda, algo, Rd, Sd, out):
    stream = cuda.cuda.current_stream()
    rc = noalloc(hj.ALGOS[algo], Rd.data_ptr(), Rd.shape[0], Sd.data_ptr(), Sd.shape[0], out.data_ptr(),
                 stream.cuda_stream)
    assert rc == 0
    stream.synchronize()
    return DeviceResult.from_buffer_copy(out.cpu().numpy().tobytes())


def test_noalloc_largest_build_and_no_device_allocation(hj, oracle, cuda):
    """A build relation of 524286 tuples (the most the fixed table takes) joins exactly, and after a
    first call per algorithm further calls leave cudaMemGetInfo's free bytes where they were."""
    noalloc = _bind(hj)
    nR = 524286
    R, S = _relations(3, nR, 1_200_000, 400_000)
    Rd = cuda.from_numpy(R.view(np.int64)).cuda()
    Sd = cuda.from_numpy(S.view(np.int64)).cuda()
    out = cuda.zeros(8, dtype=cuda.int64, device="cuda")
    want = {algo: oracle.join(algo, R, S) for algo in ("nphj_sc", "nphj_lp")}
    for algo in want:  # first calls: module load, address look-up
        got = _call(noalloc, hj, cuda, algo, Rd, Sd, out)
        assert got.error_bits == 0 and (got.matched_cnt, got.checksum) == want[algo], algo
    cuda.cuda.synchronize()
    free_before, _ = cuda.cuda.mem_get_info()
    for _ in range(3):
        for algo in want:
            got = _call(noalloc, hj, cuda, algo, Rd, Sd, out)
            assert got.error_bits == 0 and (got.matched_cnt, got.checksum) == want[algo], algo
    cuda.cuda.synchronize()
    free_after, _ = cuda.cuda.mem_get_info()
    assert free_after >= free_before, (free_before, free_after)


def test_noalloc_rejects_oversized_build(hj, cuda):
    noalloc = _bind(hj)
    out = cuda.zeros(8, dtype=cuda.int64, device="cuda")
    big = 524287
    R = cuda.ones((big, 2), dtype=cuda.int64, device="cuda")
    rc = noalloc(hj.ALGOS["nphj_sc"], R.data_ptr(), big, R.data_ptr(), 1, out.data_ptr(), None)
    assert rc == hj.HJ_E_INVAL
