"""The allocation-free join entry point (hj_nphj_join_noalloc), through the C ABI.

It exists for callers that cannot allocate device memory (an engine that owns the GPU's memory, or a
request loop that must not call the CUDA allocator): its table lives in a fixed array of the library.
Two calls in a row on different relations must each give the result of the regular entry point
(hj_join), bit for bit: the second call must not see the first call's table contents.
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


def test_noalloc_matches_regular_entry_point_twice(hj, cuda):
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


def test_noalloc_rejects_oversized_build(hj, cuda):
    noalloc = _bind(hj)
    out = cuda.zeros(8, dtype=cuda.int64, device="cuda")
    big = 524287
    R = cuda.ones((big, 2), dtype=cuda.int64, device="cuda")
    rc = noalloc(hj.ALGOS["nphj_sc"], R.data_ptr(), big, R.data_ptr(), 1, out.data_ptr(), None)
    assert rc == hj.HJ_E_INVAL
