"""CPU tests of the oracle and of the host-side generators, pinned against the reference.

Pins, in order of strength:
  1. golden fixtures produced by the reference's own generator and joins (tests/golden/
     reference_small.json, made by tests/golden/make_golden.py);
  2. the reference's published log values (closed forms, logs/*/*.log);
  3. the reference binary itself (oracle/_ref), when it has been built on this machine.
"""
import ctypes
import hashlib
import json
import os
import pathlib

def _load_oracle_module():
    import importlib.util

    root = pathlib.Path(__file__).resolve().parents[1]
    spec = importlib.util.spec_from_file_location("hj_oracle_probe", root / "oracle" / "hj_oracle.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


_REF_SOURCES = _load_oracle_module().ref_sources_present()

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
GOLDEN = json.loads((ROOT / "tests" / "golden" / "reference_small.json").read_text())


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_glibc_random_restatement_matches_libc():
    """The oracle's restated generator equals glibc's rand() after srand(seed)."""
    from conftest import load_oracle

    orc = load_oracle()
    libc = ctypes.CDLL("libc.so.6")
    for seed in (12345, 1, 0, 7, 2**31 + 5, 2**32 - 1):
        libc.srand(ctypes.c_uint(seed))
        want = [libc.rand() for _ in range(2000)]
        g = orc.GlibcRandom(seed)
        got = [g.rand() for _ in range(2000)]
        assert got == want, seed


@pytest.mark.parametrize("case", GOLDEN["cases"], ids=lambda c: c["name"])
def test_product_generator_matches_reference_bytes(hj, case):
    """hj_gen_* replays the reference generator byte for byte (sha256 of the reference's .bin files)."""
    nR, nS = case["nR"], case["nS"]
    if case["gen"] == "zipf":
        R, _ = hj.gen_pkfk_uniform(nR, nR)
        S = hj.gen_zipf(nS, nR, case["factor"])
    elif case["gen"] == "dup":
        R, S = hj.gen_dup_uniform(nR, nS)
    else:
        R, S = hj.gen_pkfk_uniform(nR, nS, payload=case["gen"] == "payload")
    assert sha(R) == case["r_sha256"]
    assert sha(S) == case["s_sha256"]


@pytest.mark.parametrize("case", [c for c in GOLDEN["cases"] if c["nS"] <= 1 << 14], ids=lambda c: c["name"])
def test_python_generator_restatement_matches_reference_bytes(oracle, case):
    """The oracle's independent Python restatement of src/gen.c gives the same bytes."""
    nR, nS = case["nR"], case["nS"]
    if case["gen"] == "zipf":
        R, _ = oracle.gen_pkfk(nR, nR)
        S = oracle.gen_zipf(nS, nR, case["factor"])
    elif case["gen"] == "dup":
        R, S = oracle.gen_dup(nR, nS)
    else:
        R, S = oracle.gen_pkfk(nR, nS, payload=case["gen"] == "payload")
    assert sha(R) == case["r_sha256"]
    assert sha(S) == case["s_sha256"]


def _golden_relations(hj, case):
    nR, nS = case["nR"], case["nS"]
    if case["gen"] == "zipf":
        R, _ = hj.gen_pkfk_uniform(nR, nR)
        return R, hj.gen_zipf(nS, nR, case["factor"])
    if case["gen"] == "dup":
        return hj.gen_dup_uniform(nR, nS)
    return hj.gen_pkfk_uniform(nR, nS, payload=case["gen"] == "payload")


@pytest.mark.parametrize("case", GOLDEN["cases"], ids=lambda c: c["name"])
def test_oracle_matches_reference_golden(hj, oracle, case):
    """Both oracle restatements reproduce every reference join result in the fixture."""
    R, S = _golden_relations(hj, case)
    for algo, (cnt, chk) in case["results"].items():
        assert oracle.join(algo, R, S) == (cnt, chk), algo
        if algo.startswith("phj"):
            c, s, rc = oracle.phj_literal(case["bits"], case["passes"], algo.endswith("lp"), R, S)
            assert rc == 0 and (c, s) == (cnt, chk), algo


# Values printed by the reference in its shipped logs (matched_cnt, check_sum).
LOG_KATS = [
    # nR, nS, matched, checksum, source
    (1 << 24, 1 << 28, 268435456, 4503599895805952, "logs/pkfkA-logs/rdx_bc_nvm.log:2"),
    (1 << 26, 1 << 28, 268435456, 18014398777917440, "logs/size-difference-logs/rdx_bc_pkfk_nvm.log:32"),
    (1 << 28, 1 << 28, 268435456, 72057594306363392, "logs/size-difference-logs/rdx_bc_pkfk_nvm.log:52"),
    (1 << 30, 1 << 34, 17179869184, 17179869184, "logs/billion-logs/rdx_bc_billion_nvm.log:12"),
]


@pytest.mark.parametrize("kat", LOG_KATS, ids=lambda k: k[4])
def test_closed_form_matches_reference_logs(hj, kat):
    nR, nS, m, c, _ = kat
    assert hj.pkfk_closed_form(nR, nS) == (m, c)


def test_closed_form_matches_oracle_small(hj, oracle):
    for nR, nS in [(256, 256), (1024, 4096), (4096, 8192)]:
        R, S = hj.gen_pkfk_uniform(nR, nS)
        assert oracle.join("phj_radix_bc", R, S) == hj.pkfk_closed_form(nR, nS)


def _random_relations(rng, nR, nS, key_range, zero_keys=False):
    R = np.empty((nR, 2), dtype=np.uint64)
    S = np.empty((nS, 2), dtype=np.uint64)
    lo = 0 if zero_keys else 1
    R[:, 0] = rng.integers(lo, key_range + 1, nR, dtype=np.uint64)
    S[:, 0] = rng.integers(lo, key_range + 1, nS, dtype=np.uint64)
    R[:, 1] = rng.integers(0, 2**64 - 1, nR, dtype=np.uint64)
    S[:, 1] = rng.integers(0, 2**64 - 1, nS, dtype=np.uint64)
    return R, S


@pytest.mark.parametrize("bits,passes", [(1, 1), (3, 1), (5, 2), (8, 1), (9, 2), (12, 2)])
def test_literal_restatement_equals_definition(oracle, bits, passes):
    """The step-by-step radix join equals the direct definition, duplicates and key 0 included."""
    rng = np.random.default_rng(bits * 10 + passes)
    for key_range, zero in [(50, False), (3000, True), (1 << 40, False)]:
        R, S = _random_relations(rng, 3000, 5000, key_range, zero)
        c, s, rc = oracle.phj_literal(bits, passes, False, R, S)
        assert rc == 0 and (c, s) == oracle.join(oracle.ALL, R, S)
        c, s, rc = oracle.phj_literal(bits, passes, True, R, S)
        if rc == 0:  # rc != 0: a full partition table with an absent key (loops in the reference)
            assert (c, s) == oracle.join(oracle.FIRST, R, S)


def test_dense_oracle_equals_hash_oracle(oracle):
    rng = np.random.default_rng(3)
    R, S = _random_relations(rng, 5000, 9000, 4000)
    for mode in (oracle.ALL, oracle.FIRST, oracle.FIRST_NP):
        assert oracle.join_dense(mode, R, S, 4000) == oracle.join(mode, R, S)


def test_key_zero_rule(oracle):
    """phj_radix_lp ignores key 0 (it marks an empty slot); nphj_lp and the all-match joins do not."""
    R = np.array([[0, 5], [1, 7], [0, 9]], dtype=np.uint64)
    S = np.array([[0, 100], [1, 200]], dtype=np.uint64)
    assert oracle.join(oracle.ALL, R, S) == (3, 5 + 100 + 9 + 100 + 7 + 200)
    assert oracle.join(oracle.FIRST, R, S) == (1, 7 + 200)
    assert oracle.join(oracle.FIRST_NP, R, S) == (2, 5 + 100 + 7 + 200)


def test_first_match_needs_order_only_for_multi_match_probes(oracle):
    """The invariant phj_radix_lp's unordered first run rests on: when no probe tuple matches two build
    tuples (key 0 never matches), the first-match result equals the all-matches result over the build
    relation without key 0, in every build order; when one does, some order changes it."""
    rng = np.random.default_rng(17)
    for case in range(6):
        nR, nS = 3000, 7000
        R = np.empty((nR, 2), dtype=np.uint64)
        R[:, 0] = rng.permutation(np.arange(1, 2 * nR + 1, dtype=np.uint64))[:nR]
        R[:, 1] = rng.integers(0, 1 << 40, nR, dtype=np.uint64)
        R[::41, 0] = 0
        if case >= 3:  # duplicate build keys; the probes of cases 3 and 4 avoid them
            R[nR // 2: nR // 2 + 50, 0] = R[1:51, 0]
        S = np.empty((nS, 2), dtype=np.uint64)
        S[:, 0] = R[rng.integers(0, nR, nS), 0]
        S[::9, 0] = 0
        S[:, 1] = rng.integers(0, 1 << 40, nS, dtype=np.uint64)
        keys, counts = np.unique(R[R[:, 0] != 0, 0], return_counts=True)
        dups = keys[counts > 1]
        if case in (3, 4):
            S = S[~np.isin(S[:, 0], dups)]
        multi = bool(np.isin(S[:, 0], dups).any())
        assert multi == (case == 5)
        nz = R[R[:, 0] != 0]
        want = oracle.join(oracle.FIRST, R, S)
        for _ in range(3):
            perm = rng.permutation(nR)
            got = oracle.join(oracle.FIRST, R[perm], S)
            if not multi:
                assert got == want == oracle.join(oracle.ALL, nz, S)
        if multi:  # reversing the build relation picks the other tuple of a probed duplicate key
            assert oracle.join(oracle.FIRST, R[::-1], S) != want


@pytest.mark.skipif(not _REF_SOURCES, reason="reference sources absent")
def test_oracle_matches_reference_binary_random(oracle):
    """Random keys with heavy duplication, straight through the reference's own joins."""
    if not (oracle.ref_available(1) and oracle.ref_available(2)):
        pytest.skip("reference not built")
    rng = np.random.default_rng(11)
    R, S = _random_relations(rng, 4096, 16384, 900)
    # Probe keys are drawn from R's keys: the reference's linear-probing joins loop forever on an absent
    # key when a table is full (src/algo/phj.c:655-658, src/algo/nphj.c:1162-1164).
    S[:, 0] = R[rng.integers(0, R.shape[0], S.shape[0]), 0]
    for algo in ("nphj_sc", "phj_radix_bc", "phj_radix_lp"):
        for bits, passes in ((6, 1), (10, 2)):
            assert oracle.ref_join(algo, R, S, bits=bits, passes=passes, threads=4) == oracle.join(algo, R, S)
    assert oracle.ref_join("nphj_lp", R, S, threads=1) == oracle.join("nphj_lp", R, S)


@pytest.mark.skipif(not _REF_SOURCES, reason="reference sources absent")
def test_reference_sc_hr_hro_and_asymm_equal_bc(oracle):
    """The reference's separate-chaining, histogram-sorted and AVX-512 partition joins, and its
    asymmetric-radix joins, return bc_join's count and checksum: the claim the library's phj_radix_sc /
    _hr / _hro and phj_asymm_radix_* names rest on. Random keys (>= 1) with heavy duplication, probe
    keys partly absent."""
    if not (oracle.ref_available(1) and oracle.ref_available(2)):
        pytest.skip("reference not built")
    rng = np.random.default_rng(12)
    R, S = _random_relations(rng, 4096, 16384, 900)
    R[:, 0] = np.maximum(R[:, 0], 1)
    S[:, 0] = np.maximum(S[:, 0], 1)
    want = oracle.join("phj_radix_bc", R, S)
    assert want[0] > S.shape[0]  # duplicates: more matches than probe tuples
    for algo in ("phj_radix_sc", "phj_radix_hr", "phj_radix_hro"):
        assert oracle.join(algo, R, S) == want
        for bits, passes in ((6, 1), (10, 2)):
            assert oracle.ref_join(algo, R, S, bits=bits, passes=passes, threads=4) == want, (algo, bits)
    # The reference's asymmetric sc and hro joins crash (SIGSEGV) or miscount on some geometries (for
    # example 12 bits over 4096 build tuples), so only its asymmetric bc and hr joins pin the split.
    R2 = R.copy()
    R2[:, 0] = rng.permutation(R.shape[0]).astype(np.uint64) + 1  # unique build keys, absent probe keys
    want2 = oracle.join("phj_radix_bc", R2, S)
    for algo in ("phj_asymm_radix_bc", "phj_asymm_radix_hr"):
        for bits, bits1 in ((10, 7), (12, 11), (8, 11), (12, 6)):
            assert oracle.ref_join(algo, R, S, bits=bits, passes=2, threads=4, bits1=bits1) == want, (algo, bits)
            assert oracle.ref_join(algo, R2, S, bits=bits, passes=2, threads=4, bits1=bits1) == want2, (algo, bits)


@pytest.mark.skipif(not _REF_SOURCES, reason="reference sources absent")
def test_reference_ptr_joins_equal_definition(hj, oracle):
    """The reference's materialising joins (pairs, then the retrieve checksum) on payload PK-FK data equal
    the definition, and so does the pairs oracle. One thread: the reference sizes each thread's pair
    buffer |S| * 1.2 / threads (src/algo/ptr_phj.h:144-145), which overflows (SIGSEGV / heap corruption)
    when the matches are spread unevenly over threads or exceed 1.2 per probe tuple."""
    if not (oracle.ref_available(1) and oracle.ref_available(2)):
        pytest.skip("reference not built")
    R, S = hj.gen_pkfk_uniform(4096, 16384, payload=True)
    for algo in ("ptr_phj_radix_bc", "ptr_phj_radix_sc", "ptr_phj_radix_hr", "ptr_phj_radix_lp", "ptr_nphj_sc",
                 "ptr_nphj_lp"):
        want = oracle.join(algo[4:], R, S)
        P = oracle.join_pairs(algo, R, S)
        assert P.shape[0] == want[0]
        assert int((P[:, 0].astype(object) + P[:, 1].astype(object)).sum()) % 2**64 == want[1]
        for bits, passes in ((6, 1), (10, 2)):
            assert oracle.ref_join(algo, R, S, bits=bits, passes=passes, threads=1) == want, (algo, bits)


@pytest.mark.skipif(os.environ.get("HJ_SLOW") != "1", reason="minutes of CPU; set HJ_SLOW=1")
def test_generator_reproduces_published_skew_and_dup_logs(hj, oracle):
    """Full-size replays of the reference's published skew/dup datasets (2^24 x 2^28)."""
    R, S = hj.gen_dup_uniform(1 << 24, 1 << 28)
    # logs/dupfk-logs/rdx_bc_dupfk_nvm.log:12
    assert oracle.join_dense(oracle.ALL, R, S, 1 << 24) == (534841984, 8973526820846944)
    del R, S
    R, _ = hj.gen_pkfk_uniform(1 << 24, 1 << 24)
    S = hj.gen_zipf(1 << 28, 1 << 24, 1.05)
    # logs/skew-logs/rdx_bc_zipf_nvm.log:12
    assert oracle.join_dense(oracle.ALL, R, S, 1 << 24) == (268435456, 38229679500325349)
