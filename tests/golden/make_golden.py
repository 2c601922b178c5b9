"""Generate tests/golden/reference_small.json by running the REFERENCE's own code (its generator and
its four joins, compiled from its sources into oracle/_ref by `make -C oracle ref`).

For each case the reference generator writes R and S (srand(seed) before each dataset, as
src/gen.c:generate_workload does); the fixture records the SHA-256 of both relation files and the
(matched_cnt, check_sum) each reference join prints. nphj_lp runs with one thread: with duplicate R keys
its multi-threaded winner is a race (src/algo/nphj.c:1064), and the single-thread outcome is the
contract. Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import importlib.util
import json
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parents[2]
spec = importlib.util.spec_from_file_location("hj_oracle", ROOT / "oracle" / "hj_oracle.py")
orc = importlib.util.module_from_spec(spec)
spec.loader.exec_module(orc)

CASES = [
    # name, generator, nR, nS, zipf factor, radix bits, passes
    ("pkfk_2e10_2e12_b4p1", "pkfk", 1 << 10, 1 << 12, None, 4, 1),
    ("pkfk_2e10_2e12_b6p2", "pkfk", 1 << 10, 1 << 12, None, 6, 2),
    ("pkfk_2e12_2e14_b14p2", "pkfk", 1 << 12, 1 << 14, None, 14, 2),
    ("payload_2e12_2e14_b10p2", "payload", 1 << 12, 1 << 14, None, 10, 2),
    ("dup_2e12_2e14_b8p1", "dup", 1 << 12, 1 << 14, None, 8, 1),
    ("dup_2e12_2e14_b11p2", "dup", 1 << 12, 1 << 14, None, 11, 2),
    ("zipf105_2e12_2e14_b10p2", "zipf", 1 << 12, 1 << 14, 1.05, 10, 2),
    ("zipf150_2e12_2e14_b7p1", "zipf", 1 << 12, 1 << 14, 1.50, 7, 1),
    ("pkfk_2e16_2e18_b14p2", "pkfk", 1 << 16, 1 << 18, None, 14, 2),
]
ALGOS = ["nphj_sc", "nphj_lp", "phj_radix_bc", "phj_radix_lp"]


def sha(a):
    return hashlib.sha256(a.tobytes()).hexdigest()


def main():
    if not orc.ref_available(1) or not orc.ref_available(2):
        sys.exit("build the reference first: make -C oracle ref")
    out = {"source": "reference sources compiled by oracle/Makefile (ref target), seed 12345", "cases": []}
    for name, kind, nR, nS, factor, bits, passes in CASES:
        if kind == "zipf":
            R, _ = orc.ref_gen("pkfk", nR, nR)
            S = orc.ref_gen("zipf", nR, nS, factor=factor)
        else:
            R, S = orc.ref_gen(kind, nR, nS)
        res = {}
        for algo in ALGOS:
            threads = 1 if algo == "nphj_lp" else 4
            res[algo] = list(orc.ref_join(algo, R, S, bits=bits, passes=passes, threads=threads))
        out["cases"].append({"name": name, "gen": kind, "nR": nR, "nS": nS, "factor": factor, "bits": bits,
                             "passes": passes, "r_sha256": sha(R), "s_sha256": sha(S), "results": res})
        print(name, res)
    (ROOT / "tests" / "golden" / "reference_small.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
