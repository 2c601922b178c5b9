"""CPU tests of the C ABI surface: the library loads and exports every function the headers declare,
name lookup follows the reference's --algo table, the host generators and .bin IO behave, and the
command-line driver mirrors bin/main and bin/gen. No kernel is launched here."""
import ctypes
import os
import subprocess

import numpy as np
import pytest


def test_every_declared_function_is_exported(hj):
    L = hj.lib()
    names = hj.header_functions()
    assert len(names) > 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


@pytest.mark.parametrize("name,code", [
    ("nphj_sc", 0), ("nphj_lp", 1), ("phj_radix_bc", 2), ("phj_radix_lp", 3), ("phj_radix_sc", 4),
    ("phj_radix_hr", 5), ("phj_radix_hro", 6), ("phj_radix_bw_reg_bc", 2), ("phj_radix_bw_reg_lp", 3),
    ("phj_radix_bw_reg_sc", 4), ("phj_radix_bw_reg_hr", 5), ("phj_radix_bw_reg_hro", 6),
    ("phj_asymm_radix_bc", 2), ("phj_asymm_radix_sc", 4), ("phj_asymm_radix_hr", 5), ("phj_asymm_radix_hro", 6),
    ("phj_asymm_radix_bw_reg_bc", 2), ("phj_asymm_radix_bw_reg_sc", 4), ("phj_asymm_radix_bw_reg_hr", 5),
    ("phj_asymm_radix_bw_reg_hro", 6)])
def test_algo_lookup(hj, name, code):
    out = ctypes.c_int(-1)
    assert hj.lib().hj_algo_from_name(name.encode(), ctypes.byref(out)) == 0
    assert out.value == code


def test_algo_lookup_unknown_and_names(hj):
    out = ctypes.c_int(-1)
    L = hj.lib()
    # names the reference does not have (src/main.c:72-143), or that this library does not implement
    for bad in (b"phj_asymm_radix_lp", b"phj_radix_bw_reg_", b"phj_radix_xx", b"ptr_phj_radix_hro", b"phj_ind_sc"):
        assert L.hj_algo_from_name(bad, ctypes.byref(out)) == hj.HJ_E_NOT_FOUND, bad
    assert L.hj_algo_from_name(None, ctypes.byref(out)) == hj.HJ_E_INVAL
    assert [L.hj_algo_name(i).decode() for i in range(7)] == ["nphj_sc", "nphj_lp", "phj_radix_bc", "phj_radix_lp",
                                                             "phj_radix_sc", "phj_radix_hr", "phj_radix_hro"]
    for code in range(10):
        assert L.hj_status_str(code)


def test_params_defaults(hj):
    p = hj.Params()
    hj.lib().hj_params_init(ctypes.byref(p))
    assert (p.num_radix_bits, p.num_passes, p.device, p.inputs_on_device, p.flags) == (14, 2, 0, 0, 0)
    assert p.table_load == 0.0  # the size-dependent default


@pytest.mark.parametrize("dup,payload", [(1, False), (1, True), (4, False)])
def test_fast_generator_distribution(hj, dup, payload):
    nR, nS = 10_000, 35_000
    R, S = hj.gen_fast_host(nR, nS, seed=5, dup=dup, payload=payload, threads=4)
    R2, S2 = hj.gen_fast_host(nR, nS, seed=5, dup=dup, payload=payload, threads=1)
    assert np.array_equal(R, R2) and np.array_equal(S, S2)  # independent of the thread count
    distinct = (nR + dup - 1) // dup
    rk = np.sort(R[:, 0])
    if dup == 1:
        assert np.array_equal(rk, np.arange(1, nR + 1, dtype=np.uint64))  # a permutation of 1..nR
    else:
        assert np.array_equal(np.bincount(rk.astype(np.int64))[1:], np.full(distinct, dup))
    counts = np.bincount(S[:, 0].astype(np.int64), minlength=distinct + 1)[1:]
    assert counts.min() >= nS // distinct and counts.max() <= nS // distinct + 1
    if payload or dup > 1:
        assert np.array_equal(S[:, 1], np.arange(1, nS + 1, dtype=np.uint64))
    else:
        assert np.array_equal(S[:, 0], S[:, 1]) and np.array_equal(R[:, 0], R[:, 1])
    R3, _ = hj.gen_fast_host(nR, nS, seed=6, dup=dup, payload=payload)
    assert not np.array_equal(R, R3)


def test_exact_generator_size_rules(hj):
    # The reference copies FK blocks of 4096 bytes and needs |S| to be a multiple of |R| (src/gen.c:178-179).
    with pytest.raises(hj.JoinError):
        hj.gen_pkfk_uniform(100, 400)
    with pytest.raises(hj.JoinError):
        hj.gen_pkfk_uniform(256, 300)


def test_closed_form(hj):
    assert hj.pkfk_closed_form(1 << 22, 1 << 23) == (8388608, 35184380477440)
    assert hj.pkfk_closed_form(1 << 27, 1 << 29) == (536870912, 72057594574798848)


def test_bin_roundtrip(hj, tmp_path):
    R, _ = hj.gen_pkfk_uniform(256, 256)
    path = str(tmp_path / "r.bin").encode()
    L = hj.lib()
    assert L.hj_store_bin(path, R.shape[0], R.ctypes.data) == 0
    assert os.path.getsize(path) == 256 * 16
    back = np.zeros_like(R)
    assert L.hj_load_bin(path, R.shape[0], back.ctypes.data) == 0
    assert np.array_equal(back, R)
    assert L.hj_load_bin(path, R.shape[0] + 1, back.ctypes.data) == hj.HJ_E_IO


def test_cli_gen_matches_library_generator(hj, tmp_path):
    r, s = tmp_path / "pk.bin", tmp_path / "fk.bin"
    out = subprocess.run([str(hj.MAIN_PATH), "--gen=pkfk", "--nr=1024", "--ns=4096", f"--out-r={r}", f"--out-s={s}"],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    R, S = hj.gen_pkfk_uniform(1024, 4096)
    assert np.array_equal(np.fromfile(r, dtype=np.uint64).reshape(-1, 2), R)
    assert np.array_equal(np.fromfile(s, dtype=np.uint64).reshape(-1, 2), S)


def test_cli_unknown_algo(hj):
    out = subprocess.run([str(hj.MAIN_PATH), "--algo=ptr_phj_radix_hro", "--r=x", "--s=y", "--nr=1", "--ns=1"],
                         capture_output=True, text=True)
    assert out.returncode == 1
    assert "does not exist" in out.stdout  # the reference's message (src/main.c:215)


def test_join_without_gpu_reports_device_error(hj):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    R = np.array([[1, 1]], dtype=np.uint64)
    r = hj.join("phj_radix_bc", R, R, check=False)
    assert r.status == hj.HJ_E_DEVICE


def test_server_without_gpu_reports_device_error(hj):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(hj.JoinError) as e:
        hj.Server(0, slots=2, hbm_budget_bytes=1e6)
    assert e.value.status == hj.HJ_E_DEVICE


def test_server_config_defaults(hj):
    L = hj._bind_server()
    cfg = hj.ServerConfig()
    assert L.hj_server_config_init(cfg) == 0
    assert (cfg.device, cfg.slots, cfg.hbm_budget_bytes, cfg.autotune) == (0, 8, 150e9, 1)
    assert (cfg.small_request_tuples, cfg.large_sm_share) == (2.0**25, 0.75)
    assert L.hj_server_config_init(None) == hj.HJ_E_INVAL
    assert 0 < hj.now()


def test_reference_table_names_resolve(hj):
    # Every name of the reference-facing dispatch table is also a library algorithm, and both agree
    # with the Python table.
    L = hj.lib()
    import ctypes as C

    class AlgoT(C.Structure):
        _fields_ = [("name", C.c_char * 128), ("fn", C.c_void_p)]

    n = C.c_int.in_dll(L, "hj_ref_algo_count").value
    table = (AlgoT * n).in_dll(L, "hj_ref_algos")
    names = [t.name.decode() for t in table]
    assert len(names) == len(set(names)) == 30
    for name in names:
        # ptr_* names are the materialising entry point (hj_join_mat) over their base algorithm
        base = name[4:] if name.startswith("ptr_") else name
        out = C.c_int(-1)
        assert L.hj_algo_from_name(base.encode(), C.byref(out)) == 0, name
        assert hj.ALGOS[base] == out.value, name
        assert getattr(L, name)  # exported under the reference's name
    assert sum(n.startswith("ptr_") for n in names) == 10


def test_python_flag_constants_match_header(hj):
    # The ctypes binding's flag values are the C header's #defines.
    import re
    text = (hj.HERE.parent / "include" / "hjscm.h").read_text()
    defs = {m.group(1): int(m.group(2), 16) for m in re.finditer(r"#define (HJ_F_\w+)\s+0x([0-9a-fA-F]+)u", text)}
    assert {"HJ_F_SEGMENTS", "HJ_F_EXACT", "HJ_F_PHASE_TIMES", "HJ_F_TEST_STALL", "HJ_F_ORDERED"} <= set(defs)
    for name, value in defs.items():
        if hasattr(hj, name):
            assert getattr(hj, name) == value, name
    assert len(set(defs.values())) == len(defs)  # no two flags share a bit
    res = {m.group(1): int(m.group(2), 16) for m in re.finditer(r"#define (HJ_RES_\w+)\s+0x([0-9a-fA-F]+)u", text)}
    assert {"HJ_RES_COMPACT_PARTITIONS", "HJ_RES_WORD_PASS1", "HJ_RES_ORDERED_PASSES"} <= set(res)
    for name, value in res.items():
        assert getattr(hj, name) == value, name
    assert len(set(res.values())) == len(res)
