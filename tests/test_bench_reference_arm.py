"""CPU tests of bench.py's reference arm: it times the reference's own join on relations that the
oracle's numpy restatement of the library's parallel generator writes, and it never loads the
library (libhjscm.so) into its process."""
import json
import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


@pytest.mark.parametrize("shape", [(1000, 3000, 0, 1), (4096, 16384, 0, 1), (4096, 12293, 1, 1),
                                   (1 << 16, 1 << 18, 0, 4), (1, 5, 0, 1), (777, 0, 0, 1), (3, 3, 1, 2)])
def test_oracle_fast_generator_equals_library_bytes(hj, oracle, shape):
    nR, nS, payload, dup = shape
    want = hj.gen_fast_host(nR, nS, seed=12345, payload=bool(payload), dup=dup)
    got = oracle.gen_fast(nR, nS, seed=12345, payload=bool(payload), dup=dup, threads=3)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_oracle_closed_form_equals_library(hj, oracle):
    for nR, nS in ((1 << 27, 1 << 29), (1 << 22, 1 << 23), (256, 256 * 16), (1 << 30, 1 << 34)):
        assert oracle.pkfk_closed_form(nR, nS) == hj.pkfk_closed_form(nR, nS)


_CHILD = r"""
import importlib.util, json, pathlib, sys
root = pathlib.Path(sys.argv[1])
spec = importlib.util.spec_from_file_location("bench", root / "bench.py")
bench = importlib.util.module_from_spec(spec)
spec.loader.exec_module(bench)
sys.argv = ["bench.py", "--impl", "reference", "--nr-log", "16", "--ns-log", "18", "--steps", "2",
            "--warmup", "2"]
assert bench.run_reference_arm(bench.parse_args(), 0, 1) == 0
maps = pathlib.Path("/proc/self/maps").read_text()
print(json.dumps({"maps_libhjscm": "libhjscm" in maps, "pkg_imported": "hashjoin_scm_b200" in sys.modules}))
"""


def test_reference_arm_runs_without_the_library(oracle):
    if not oracle.ref_available(2):
        if not oracle.ref_build():
            pytest.skip("reference binary not built (no reference sources)")
    out = subprocess.run([sys.executable, "-c", _CHILD, str(ROOT)], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]
    ref_line, probe = lines[0], lines[-1]
    assert probe == {"maps_libhjscm": False, "pkg_imported": False}
    assert ref_line["impl"] == "reference" and ref_line["warmup"] == 2 and ref_line["steps"] == 2
    assert ref_line["cpu_baseline"]["kind"] == "reference" and ref_line["value"] > 0
    assert ref_line["e2e"]["h2d_bytes_per_step"] == 0
