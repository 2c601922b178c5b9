"""The drop-in boundary, shown with the reference's own driver: src/main.c, compiled unchanged (with
the reference's src/inc/utils.c) and linked against libhjscm.so by oracle/Makefile (target refmain,
binary oracle/_ref/hjref_main). The driver reads a workload file with the reference's data_cfg,
looks the --algo name up in its own table (src/main.c:70-220) and calls the library's entry point of
that name, then prints its per-trial and averaged lines (src/main.c:429-459).

CPU tests: the driver parses workload files and dispatches names (out-of-scope names reach the stub
that says so). GPU tests: each in-scope name prints the oracle's matched_cnt / check_sum on every
trial, and the averaged line over the two timed trials."""
import os
import pathlib
import re
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
BIN = ROOT / "oracle" / "_ref" / "hjref_main"

pytestmark = pytest.mark.skipif(not BIN.exists(), reason="oracle/_ref/hjref_main not built (no reference sources)")

CFG = """r_path_suffix = "{sub}/pk_R.bin";
s_path_suffix = "{sub}/fk_S.bin";

r_tuple_num = {nR};
s_tuple_num = {nS};
r_tuple_size = 16;
s_tuple_size = 16;

theta = 0.0;
selectivity = 1.0;
density = 1.0;
sparsity = 1.0;

min_key = 1;
max_key = {nR};

workload_name = "{sub}_pkfk_{tag}";
"""


def workload(tmp, R, S, sub="uniform", tag="T"):
    (tmp / "bins" / sub).mkdir(parents=True, exist_ok=True)
    (tmp / "data" / sub).mkdir(parents=True, exist_ok=True)
    R.tofile(tmp / "bins" / sub / "pk_R.bin")
    S.tofile(tmp / "bins" / sub / "fk_S.bin")
    (tmp / "data" / sub / f"pkfk_{tag}.cfg").write_text(CFG.format(sub=sub, nR=R.shape[0], nS=S.shape[0], tag=tag))
    (tmp / "cpu.cfg").write_text("cores: {\n  local_core_id_arrays = [0, 1, 2, 3];\n"
                                 "  remote_core_id_arrays = [4, 5, 6, 7];\n};\n")


def run(tmp, algo, sub="uniform", tag="T", extra_env=None):
    env = dict(os.environ, HJ_DATA_PATH_PREFIX=str(tmp / "bins"), HJREF_CFG_PREFIX=str(tmp),
               HJREF_CPU_CFG=str(tmp / "cpu.cfg"), HJREF_WORK_PREFIX=str(tmp), **(extra_env or {}))
    out = subprocess.run([str(BIN), f"--algo={algo}", f"--workload={sub}", f"--subtype={tag}", "--param=pkfk"],
                         capture_output=True, text=True, timeout=300, env=env, cwd=tmp)
    return out.returncode, re.sub(r"\x1b\[[0-9;]*m", "", out.stdout), out.stderr


TRIAL = re.compile(r"^memory_type: dram\talgo: (\S+)\tworkload: (\S+)\tbuildpart_time: ([-\d.]+)\t"
                   r"probejoin_time: ([-\d.]+)\ttotal_time: ([-\d.]+)", re.M)
AVG = re.compile(r"num_trials: (\d+)\tmemory_type: dram\talgo: (\S+)\tworkload: (\S+)\t.*total_time: ([-\d.]+)")
RESULT = re.compile(r"matched_cnt: (\d+)\tcheck_sum: (\d+)")


def test_driver_parses_workload_and_dispatches_out_of_scope_names(tmp_path, hj):
    R, S = hj.gen_pkfk_uniform(1 << 10, 1 << 12)
    workload(tmp_path, R, S)
    rc, out, _ = run(tmp_path, "eth_pro")
    assert rc == 0
    assert out.count("eth_pro is not provided by this library") == 3  # TRIAL_NUM trials
    trials = TRIAL.findall(out)
    assert len(trials) == 3 and all(t[0] == "eth_pro" and t[1] == "uniform_pkfk_T" for t in trials)
    avg = AVG.findall(out)
    assert avg and avg[0][0] == "2" and avg[0][1] == "eth_pro"
    rc, out, _ = run(tmp_path, "no_such_join")
    assert rc != 0 and "does not exist" in out


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ["phj_radix_bc", "phj_radix_lp", "nphj_sc", "nphj_lp", "phj_radix_hr",
                                  "phj_asymm_radix_bc", "phj_radix_bw_reg_bc", "ptr_phj_radix_bc", "ptr_nphj_sc"])
def test_reference_driver_runs_library_joins(tmp_path, hj, oracle, cuda, algo):
    if algo.startswith("ptr_"):
        R, S = hj.gen_pkfk_uniform(1 << 12, 1 << 14, payload=True)  # retrieve needs row id = position
    else:
        R, S = hj.gen_dup_uniform(1 << 12, 1 << 14)  # duplicate keys: bc and lp results differ
    workload(tmp_path, R, S)
    rc, out, err = run(tmp_path, algo)
    assert rc == 0, err
    want = oracle.join(algo.replace("ptr_", ""), R, S)
    results = [(int(a), int(b)) for a, b in RESULT.findall(out)]
    assert results == [want] * 3, (results, want)
    trials = TRIAL.findall(out)
    assert len(trials) == 3 and all(float(t[4]) > 0 for t in trials)
    avg = AVG.findall(out)
    assert avg and avg[0][0] == "2" and avg[0][1] == algo and float(avg[0][3]) > 0


@pytest.mark.gpu
def test_reference_driver_config1_workload(tmp_path, hj, cuda):
    """The reference's C1 shape (nphj_sc, 2^22 x 2^23, the reference generator's bytes) through the
    reference's driver: the closed form 8388608 / 35184380477440 on every trial."""
    R, S = hj.gen_fast_host(1 << 22, 1 << 23)
    workload(tmp_path, R, S, tag="C1")
    rc, out, err = run(tmp_path, "nphj_sc", tag="C1")
    assert rc == 0, err
    assert [(int(a), int(b)) for a, b in RESULT.findall(out)] == [hj.pkfk_closed_form(1 << 22, 1 << 23)] * 3
