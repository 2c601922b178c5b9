"""GPU parity: every join on the B200 against the oracle and the reference's golden values, through
the C ABI (libhjscm.so). Integer results must match bit for bit."""
import json
import pathlib

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
GOLDEN = json.loads((ROOT / "tests" / "golden" / "reference_small.json").read_text())
ALGOS = ["nphj_sc", "nphj_lp", "phj_radix_bc", "phj_radix_lp"]
U64MAX = np.uint64(2**64 - 1)

pytestmark = pytest.mark.gpu


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def run(hj, algo, R, S, cuda=None, **kw):
    if cuda is not None:
        r = hj.join(algo, dev(cuda, R), dev(cuda, S), on_device=True, **kw)
    else:
        r = hj.join(algo, R, S, **kw)
    return r.matched_cnt, r.checksum


def golden_relations(hj, case):
    nR, nS = case["nR"], case["nS"]
    if case["gen"] == "zipf":
        R, _ = hj.gen_pkfk_uniform(nR, nR)
        return R, hj.gen_zipf(nS, nR, case["factor"])
    if case["gen"] == "dup":
        return hj.gen_dup_uniform(nR, nS)
    return hj.gen_pkfk_uniform(nR, nS, payload=case["gen"] == "payload")


@pytest.mark.parametrize("case", GOLDEN["cases"], ids=lambda c: c["name"])
def test_golden_reference_results(hj, cuda, case):
    R, S = golden_relations(hj, case)
    for algo in ALGOS:
        want = tuple(case["results"][algo])
        got_host = run(hj, algo, R, S, bits=case["bits"], passes=case["passes"])
        got_dev = run(hj, algo, R, S, cuda, bits=case["bits"], passes=case["passes"])
        assert got_host == want, (algo, "host inputs")
        assert got_dev == want, (algo, "device inputs")


def random_rel(rng, n, lo, hi):
    a = np.empty((n, 2), dtype=np.uint64)
    a[:, 0] = rng.integers(lo, hi, n, dtype=np.uint64, endpoint=True)
    a[:, 1] = rng.integers(0, 2**64 - 1, n, dtype=np.uint64, endpoint=True)
    return a


@pytest.mark.parametrize("bits,passes", [(1, 1), (4, 1), (8, 1), (9, 1), (3, 2), (10, 2), (14, 2), (15, 2), (14, 1)])
def test_radix_geometries(hj, oracle, cuda, bits, passes):
    rng = np.random.default_rng(bits * 3 + passes)
    R = random_rel(rng, 50_000, 1, 200_000)
    S = random_rel(rng, 120_000, 1, 200_000)  # about a quarter of the probes find a key
    for algo in ("phj_radix_bc", "phj_radix_lp"):
        assert run(hj, algo, R, S, cuda, bits=bits, passes=passes) == oracle.join(algo, R, S), algo


@pytest.mark.parametrize("algo", ALGOS)
def test_edge_cases(hj, oracle, cuda, algo):
    rng = np.random.default_rng(5)
    one = np.array([[7, 70]], dtype=np.uint64)
    other = np.array([[8, 80]], dtype=np.uint64)
    empty = np.zeros((0, 2), dtype=np.uint64)
    cases = [
        (empty, one), (one, empty), (empty, empty),
        (one, one), (one, other),
        (random_rel(rng, 1000, 1, 3000), random_rel(rng, 3333, 1, 3000)),     # ragged sizes
        (random_rel(rng, 4097, 1, 10**12), random_rel(rng, 7001, 1, 10**12)),  # almost no matches
        (random_rel(rng, 5000, 1, 60), random_rel(rng, 9000, 1, 80)),          # heavy duplicates
        (random_rel(rng, 3000, 0, 5), random_rel(rng, 3000, 0, 6)),            # key 0 present
    ]
    for R, S in cases:
        want = oracle.join(algo, R, S)
        assert run(hj, algo, R, S) == want, (algo, R.shape, S.shape)
        if R.shape[0] and S.shape[0]:
            assert run(hj, algo, R, S, cuda) == want, (algo, "device")


@pytest.mark.parametrize("algo", ALGOS)
def test_all_ones_key(hj, oracle, cuda, algo):
    """Key 2^64-1 is the NPHJ table's empty pattern; it still joins like any other key."""
    rng = np.random.default_rng(9)
    R = random_rel(rng, 2000, 1, 500)
    S = random_rel(rng, 4000, 1, 500)
    R[::97, 0] = U64MAX
    S[::31, 0] = U64MAX
    assert run(hj, algo, R, S, cuda) == oracle.join(algo, R, S)


@pytest.mark.parametrize("algo", ["phj_radix_bc", "phj_radix_lp"])
def test_large_partitions(hj, oracle, cuda, algo):
    """Build partitions beyond the shared-memory capacity take the global-memory path."""
    rng = np.random.default_rng(21)
    n = 60_000
    R = np.empty((n, 2), dtype=np.uint64)
    # Every key in partition 3 of 2^14: |R_p| = 60000 > the shared-memory capacity.
    R[:, 0] = (rng.integers(1, 40_000, n, dtype=np.uint64) << np.uint64(14)) | np.uint64(3)
    R[:, 1] = np.arange(n, dtype=np.uint64)
    S = R[rng.integers(0, n, 150_000)].copy()
    S[:, 1] = np.arange(S.shape[0], dtype=np.uint64) * np.uint64(3)
    S[::7, 0] += np.uint64(1 << 14)  # some probes miss
    r = hj.join(algo, dev(cuda, R), dev(cuda, S), on_device=True, bits=14, passes=2)
    assert (r.matched_cnt, r.checksum) == oracle.join(algo, R, S)
    assert r.large_partitions >= 1


@pytest.mark.parametrize("factor", [0.5, 1.0, 1.5])
def test_zipf_probe_side(hj, oracle, cuda, factor):
    """Skewed probe side: a few partitions hold most of S and are split into several work items."""
    nR, nS = 1 << 16, 1 << 21
    R, _ = hj.gen_fast_host(nR, nR, seed=7)
    S = cuda.empty((nS, 2), dtype=cuda.int64, device="cuda")
    hj.gen_zipf_device(nS, nR, factor, S.data_ptr(), seed=7)
    cuda.cuda.synchronize()
    S_host = S.cpu().numpy().view(np.uint64)
    for algo in ALGOS:
        want = oracle.join(algo, R, S_host)
        got = hj.join(algo, dev(cuda, R), S, on_device=True)
        assert (got.matched_cnt, got.checksum) == want, algo


def test_dup_variant(hj, oracle, cuda):
    """R keys repeated 4x (the dup-FK configuration shape), uniform probes."""
    nR, nS = 1 << 18, 1 << 20
    R, S = hj.gen_fast_host(nR, nS, seed=3, dup=4)
    for algo in ALGOS:
        assert run(hj, algo, R, S, cuda) == oracle.join(algo, R, S), algo


def test_fast_generator_host_equals_device(hj, cuda):
    for nR, nS, dup, payload in [(1000, 3000, 1, False), (1 << 16, 1 << 18, 1, True), (4096, 10000, 4, False)]:
        R, S = hj.gen_fast_host(nR, nS, seed=99, dup=dup, payload=payload)
        Rd = cuda.empty((nR, 2), dtype=cuda.int64, device="cuda")
        Sd = cuda.empty((nS, 2), dtype=cuda.int64, device="cuda")
        hj.gen_fast_device(nR, nS, Rd.data_ptr(), Sd.data_ptr(), seed=99, dup=dup, payload=payload)
        cuda.cuda.synchronize()
        assert np.array_equal(Rd.cpu().numpy().view(np.uint64), R)
        assert np.array_equal(Sd.cpu().numpy().view(np.uint64), S)


def test_config1_nphj_sc_exact_generator(hj, cuda):
    """nphj_sc on R = 2^22, S = 2^23 from the reference's generator: closed-form result."""
    R, S = hj.gen_pkfk_uniform(1 << 22, 1 << 23)
    want = hj.pkfk_closed_form(1 << 22, 1 << 23)
    assert want == (8388608, 35184380477440)
    for algo in ALGOS:
        assert run(hj, algo, R, S, cuda) == want, algo


def test_config2_full_size_closed_form(hj, cuda):
    """phj_radix_bc 2^27 x 2^29, 14 bits, 2 passes: the size-independent closed form holds."""
    nR, nS = 1 << 27, 1 << 29
    R = cuda.empty((nR, 2), dtype=cuda.int64, device="cuda")
    S = cuda.empty((nS, 2), dtype=cuda.int64, device="cuda")
    hj.gen_fast_device(nR, nS, R.data_ptr(), S.data_ptr(), seed=12345)
    cuda.cuda.synchronize()
    want = hj.pkfk_closed_form(nR, nS)
    assert want == (536870912, 72057594574798848)
    for algo in ("phj_radix_bc", "phj_radix_lp"):
        r = hj.join(algo, R, S, on_device=True, bits=14, passes=2)
        assert (r.matched_cnt, r.checksum) == want, algo
        assert r.large_partitions == 0
    del R, S
    cuda.cuda.empty_cache()


def test_invalid_arguments(hj):
    R = np.array([[1, 1]], dtype=np.uint64)
    r = hj.join("phj_radix_bc", R, R, bits=16, check=False)
    assert r.status == hj.HJ_E_INVAL
    r = hj.join("phj_radix_bc", R, R, passes=3, check=False)
    assert r.status == hj.HJ_E_INVAL


def test_context_reuse_is_deterministic(hj, oracle, cuda):
    rng = np.random.default_rng(77)
    R = random_rel(rng, 100_000, 1, 70_000)
    S = random_rel(rng, 300_000, 1, 70_000)
    want = {a: oracle.join(a, R, S) for a in ALGOS}
    with hj.Context(0) as ctx:
        for _ in range(3):
            for a in ALGOS:
                r = hj.join(a, R, S, ctx=ctx)
                assert (r.matched_cnt, r.checksum) == want[a]


@pytest.mark.parametrize("wide_fields", [False, True])
@pytest.mark.parametrize("algo", ["phj_radix_bc", "phj_radix_lp"])
def test_mixed_partition_sizes(hj, oracle, cuda, algo, wide_fields):
    """Partitions below the compact table's capacity, between it and the shared-memory capacity, and
    above it (global-memory path) in one join; with 32-bit-fitting keys/row ids (compact table used)
    and with 64-bit ones (compact table not applicable)."""
    rng = np.random.default_rng(31 + wide_fields)
    sizes = {0: 5000, 1: 9000, 2: 9800, 3: 20000}  # partition (key & 3) -> |R_p|
    parts = []
    for p, n in sizes.items():
        hi = rng.permutation(4 * n)[:n].astype(np.uint64) + np.uint64(1)
        parts.append((hi << np.uint64(2)) | np.uint64(p))
    keys = np.concatenate(parts)
    if wide_fields:
        keys = keys | np.uint64(1 << 62)
    R = np.empty((keys.shape[0], 2), dtype=np.uint64)
    R[:, 0] = rng.permutation(keys)
    R[:, 1] = rng.integers(0, 2**63 if wide_fields else 2**31, R.shape[0], dtype=np.uint64)
    R[::50, 0] = R[1::50, 0]  # some duplicate build keys
    S = R[rng.integers(0, R.shape[0], 200_000)].copy()
    S[:, 1] = rng.integers(0, 2**31, S.shape[0], dtype=np.uint64)
    S[::9, 0] += np.uint64(4)  # misses in the same partition
    got = run(hj, algo, R, S, cuda, bits=2, passes=1)
    assert got == oracle.join(algo, R, S)


@pytest.mark.parametrize("algo", ["phj_radix_bc", "phj_radix_lp"])
def test_many_subchunks_with_duplicates(hj, oracle, cuda, algo):
    # 2^22 + 2^24 tuples make chunks of 24 tiles, i.e. two pass-1 work items per chunk (16 tiles and a
    # partial 8), plus a ragged last chunk; duplicate build keys make the lp result depend on order.
    rng = np.random.default_rng(31)
    nR, nS = (1 << 22) + 777, (1 << 24) - 1234
    R = np.empty((nR, 2), dtype=np.uint64)
    S = np.empty((nS, 2), dtype=np.uint64)
    R[:, 0] = rng.integers(0, 1 << 20, nR, dtype=np.uint64)
    R[:, 1] = rng.integers(0, 2**48, nR, dtype=np.uint64)
    S[:, 0] = rng.integers(0, (1 << 20) + 4096, nS, dtype=np.uint64)
    S[:, 1] = rng.integers(0, 2**48, nS, dtype=np.uint64)
    want = oracle.join(algo, R, S)
    assert run(hj, algo, R, S, cuda) == want
    assert run(hj, algo, R, S, cuda, bits=11, passes=2) == want


@pytest.mark.parametrize("algo", ["phj_radix_sc", "phj_radix_hr", "phj_radix_hro", "phj_radix_bw_reg_hro",
                                  "phj_asymm_radix_bc", "phj_asymm_radix_sc", "phj_asymm_radix_hr",
                                  "phj_asymm_radix_bw_reg_hro"])
def test_every_match_family(hj, oracle, cuda, algo):
    # sc / hr / hro and the asymmetric names count every match, as bc does; every bit split (requested
    # pass-1 bits are clamped to the split where each pass has 1..8 bits) gives the same partitions.
    rng = np.random.default_rng(41)
    nR, nS = 30_000, 90_000
    R = np.empty((nR, 2), dtype=np.uint64)
    S = np.empty((nS, 2), dtype=np.uint64)
    R[:, 0] = rng.integers(0, 6000, nR, dtype=np.uint64)
    S[:, 0] = rng.integers(0, 7000, nS, dtype=np.uint64)
    R[:, 1] = rng.integers(0, 2**64 - 1, nR, dtype=np.uint64)
    S[:, 1] = rng.integers(0, 2**64 - 1, nS, dtype=np.uint64)
    R[::97, 0] = U64MAX
    S[::89, 0] = U64MAX
    want = oracle.join("phj_radix_bc", R, S)
    for bits, passes, b1 in ((14, 2, None), (14, 2, 8), (14, 2, 3), (10, 2, 11), (9, 2, 1), (6, 1, None)):
        assert run(hj, algo, R, S, cuda, bits=bits, passes=passes, bits_pass1=b1) == want, (bits, passes, b1)


def test_asymm_cli_entry_point(hj, tmp_path):
    # The reference-named entry point phj_asymm_radix_hr through the bin/main-style driver, with the
    # pass-1 bits from the environment as the reference's NUM_RADIX_BITS_PASS1.
    import os
    import subprocess

    R, S = hj.gen_dup_uniform(1 << 12, 1 << 14)
    R.tofile(tmp_path / "r.bin")
    S.tofile(tmp_path / "s.bin")
    env = dict(os.environ, HJ_NUM_RADIX_BITS_PASS1="7", HJ_NUM_RADIX_BITS="12")
    out = subprocess.run([str(hj.MAIN_PATH), "--algo=phj_asymm_radix_hr", f"--r={tmp_path / 'r.bin'}",
                          f"--s={tmp_path / 's.bin'}",
                          f"--nr={1 << 12}", f"--ns={1 << 14}"], capture_output=True, text=True, env=env)
    assert out.returncode == 0, out.stderr
    want = hj.join("phj_radix_bc", R, S)
    assert f"matched_cnt: {want.matched_cnt}\tcheck_sum: {want.checksum}" in out.stdout


def test_cli_workload_config_files(hj, tmp_path):
    # bin/main's way of naming a workload: --workload/--subtype/--param select
    # $HJ_DATA_CFG_PATH_PREFIX/data/<workload>/<param>_<subtype>.cfg, whose path suffixes are read under
    # $HJ_DATA_PATH_PREFIX; per-trial and averaged lines as src/main.c:439-459 prints them.
    import os
    import subprocess

    nR, nS = 1 << 12, 1 << 14
    R, S = hj.gen_pkfk_uniform(nR, nS, payload=True)
    (tmp_path / "data" / "t").mkdir(parents=True)
    (tmp_path / "rel" / "t").mkdir(parents=True)
    R.tofile(tmp_path / "rel" / "t" / "pk_TR.bin")
    S.tofile(tmp_path / "rel" / "t" / "fk_TS.bin")
    (tmp_path / "data" / "t" / "pkfk_T.cfg").write_text(
        'r_path_suffix = "t/pk_TR.bin";\ns_path_suffix = "t/fk_TS.bin";\n\n'
        f"r_tuple_num = {nR};\ns_tuple_num = {nS};\nr_tuple_size = 16;\ns_tuple_size = 16;\n\n"
        "theta = 0.0;\nselectivity = 1.0;\ndensity = 1.0;\nsparsity = 1.0;\n\n"
        f'min_key = 1;\nmax_key = {nR};\n\nworkload_name = "test_pkfk_T";\n')
    env = dict(os.environ, HJ_DATA_CFG_PATH_PREFIX=str(tmp_path), HJ_DATA_PATH_PREFIX=str(tmp_path / "rel"))
    want = hj.join("phj_radix_bc", R, S)
    for algo in ("phj_radix_bc", "ptr_phj_radix_bc", "nphj_lp"):
        out = subprocess.run([str(hj.MAIN_PATH), f"--algo={algo}", "--workload=t", "--subtype=T", "--param=pkfk",
                              "--trials=3"], capture_output=True, text=True, env=env)
        assert out.returncode == 0, out.stdout + out.stderr
        assert out.stdout.count(f"matched_cnt: {want.matched_cnt}\tcheck_sum: {want.checksum}") == 3
        trial_lines = [ln for ln in out.stdout.splitlines() if ln.startswith("memory_type: HBM\talgo: " + algo)]
        assert len(trial_lines) == 3 and all("\tworkload: test_pkfk_T\t" in ln for ln in trial_lines)
        assert "num_trials: 2\t" in out.stdout
