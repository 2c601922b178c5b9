"""CPU oracle for the equi-join hot path - TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker; the product
(hashjoin-scm_b200/) never imports it.

Contents
- GlibcRandom: restatement of glibc's default random()/rand() generator (TYPE_3 additive feedback,
  r[i] = r[i-3] + r[i-31] mod 2^32, output r >> 1, seeded by the 16807 LCG with 310 discards), the
  generator the reference's bin/gen draws from after srand(12345) (src/gen.c:144).
- gen_pkfk / gen_dup / gen_zipf: pure-Python restatements of src/gen.c:161-331 and
  src/inc/eth_genzipf.c:31-147 on top of GlibcRandom (small sizes only: they are Python loops).
- join / phj_literal / join_dense: ctypes front-ends of hj_oracle.c (the C restatement of the joins).
- ref_*: run the reference's own code (built from its sources by oracle/Makefile into oracle/_ref).
"""
from __future__ import annotations

import ctypes
import math
import os
import pathlib
import re
import subprocess
import tempfile

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"

ALL, FIRST, FIRST_NP = 0, 1, 2  # hj_oracle.c modes: bc/sc, phj lp, nphj lp
# sc_join, hr_join and hro_join count every match (src/algo/phj.c:683-1037), as bc_join does.
MODE_OF_ALGO = {"nphj_sc": ALL, "phj_radix_bc": ALL, "nphj_lp": FIRST_NP, "phj_radix_lp": FIRST,
                "phj_radix_sc": ALL, "phj_radix_hr": ALL, "phj_radix_hro": ALL}
for _s, _m in (("bc", ALL), ("lp", FIRST), ("sc", ALL), ("hr", ALL), ("hro", ALL)):
    MODE_OF_ALGO["phj_radix_bw_reg_" + _s] = _m
    if _s != "lp":
        MODE_OF_ALGO["phj_asymm_radix_" + _s] = _m
        MODE_OF_ALGO["phj_asymm_radix_bw_reg_" + _s] = _m
RAND_MAX = 2147483647
MASK64 = (1 << 64) - 1


# ------------------------------------------------------------------------------------------------
# glibc random()
# ------------------------------------------------------------------------------------------------
class GlibcRandom:
    """glibc random_r with the default 128-byte state (TYPE_3: degree 31, separation 3)."""

    def __init__(self, seed: int):
        seed &= 0xFFFFFFFF
        if seed == 0:
            seed = 1
        r = [0] * 31
        r[0] = seed
        word = seed if seed < 2**31 else seed - 2**32
        for i in range(1, 31):
            hi, lo = divmod(word, 127773) if word >= 0 else (-((-word) // 127773), -((-word) % 127773))
            word = 16807 * lo - 2836 * hi
            if word < 0:
                word += 2147483647
            r[i] = word & 0xFFFFFFFF
        self.r = r
        self.f = 3  # front pointer index
        self.b = 0  # rear pointer index
        for _ in range(310):
            self._step()

    def _step(self) -> int:
        r = self.r
        r[self.f] = (r[self.f] + r[self.b]) & 0xFFFFFFFF
        out = r[self.f] >> 1
        self.f = (self.f + 1) % 31
        self.b = (self.b + 1) % 31
        return out

    def rand(self) -> int:
        return self._step()


# ------------------------------------------------------------------------------------------------
# Generator restatements (src/gen.c, src/inc/eth_genzipf.c)
# ------------------------------------------------------------------------------------------------
def _knuth_shuffle(g: GlibcRandom, t: np.ndarray) -> None:
    """src/gen.c:161-171: for i in 0..n-1: j = rand() % n; swap(t[i], t[j])."""
    n = t.shape[0]
    for i in range(n):
        j = g.rand() % n
        if i != j:
            tmp = t[j].copy()
            t[j] = t[i]
            t[i] = tmp


def gen_pkfk(nR: int, nS: int, seed: int = 12345, payload: bool = False):
    """gen_pkfk_uniform (src/gen.c:199-223) / payload_gen_pkfk_uniform (src/gen.c:258-283)."""
    assert nS % nR == 0 and (nR * 16) % 4096 == 0
    g = GlibcRandom(seed)
    R = np.empty((nR, 2), dtype=np.uint64)
    R[:, 0] = np.arange(1, nR + 1, dtype=np.uint64)
    R[:, 1] = R[:, 0]
    _knuth_shuffle(g, R)
    S = np.concatenate([R] * (nS // nR))  # gen_fk_from_pk copies (src/gen.c:178-182)
    _knuth_shuffle(g, S)
    if payload:
        S[:, 1] = np.arange(1, nS + 1, dtype=np.uint64)
        R[:, 1] = np.arange(1, nR + 1, dtype=np.uint64)
    return R, S


def gen_dup(nR: int, nS: int, seed: int = 12345):
    """gen_dup_uniform (src/gen.c:286-331)."""
    assert nS % nR == 0 and (nR * 16) % 4096 == 0
    g = GlibcRandom(seed)
    uni = g.rand() % RAND_MAX
    R = np.empty((nR, 2), dtype=np.uint64)
    for i in range(nR):
        k = int(uni / 127773) if uni >= 0 else -int(-uni / 127773)
        uni = 16807 * (uni - k * 127773) - k * 2836
        # the reference computes this in 32-bit int arithmetic
        uni = ((uni + 2**31) % 2**32) - 2**31
        if uni < 0:
            uni += 2147483647
        r = uni * 4.656612875e-10
        r = (1.0 - r) * (1 - 0.5) + r * (nR + 0.5)
        key = int(_c_round(r))
        key = min(max(key, 1), nR)
        R[i, 0] = key
        R[i, 1] = i + 1
    _knuth_shuffle(g, R)
    S = np.concatenate([R] * (nS // nR))
    _knuth_shuffle(g, S)
    return R, S


def _c_round(x: float) -> float:
    """C round(): half away from zero."""
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)


def gen_zipf(nS: int, nR: int, factor: float, seed: int = 12345):
    """gen_zipf (src/inc/eth_genzipf.c:97-147) after gen_alphabet and gen_zipf_lut."""
    g = GlibcRandom(seed)
    alphabet = list(range(1, nR + 1))
    for i in range(nR - 1, 0, -1):
        k = (i * g.rand()) // RAND_MAX
        alphabet[i], alphabet[k] = alphabet[k], alphabet[i]
    scale = 0.0
    for i in range(1, nR + 1):
        scale += 1.0 / math.pow(i, factor)
    lut = []
    s = 0.0
    for i in range(1, nR + 1):
        s += 1.0 / math.pow(i, factor)
        lut.append(s / scale)
    S = np.empty((nS, 2), dtype=np.uint64)
    for j in range(nS):
        r = g.rand() / RAND_MAX
        if lut[0] >= r:
            pos = 0
        else:
            left, right = 1, nR
            while right - left > 1:
                m = (left + right) // 2
                if lut[m] < r:
                    left = m
                else:
                    right = m
            pos = right
        S[j, 0] = alphabet[pos]
        S[j, 1] = j + 1
    return S


# ------------------------------------------------------------------------------------------------
# The library's parallel PK-FK generator (hj_gen_fast_host / hj_gen_fast_device), restated in numpy
# so that the CPU-baseline leg of the benchmark can write the same relations without loading the
# library. The reference draws its permutation with a sequential Knuth shuffle (src/gen.c:161-171);
# the library replaces that shuffle by a keyed bijection of [0, n): a 6-round unbalanced Feistel
# network over the smallest power of two >= n (round function: the splitmix64 output mix of Steele,
# Lea and Flood, 2014), with cycle walking back into [0, n). R tuple i = perm_R(i) + 1 (mod the
# distinct-key count for the duplicate variant); S tuple j = perm_S(j) mod |distinct| + 1.
# ------------------------------------------------------------------------------------------------
_GOLDEN = 0x9E3779B97F4A7C15


def _mix64_int(z: int) -> int:
    z ^= z >> 30
    z = (z * 0xBF58476D1CE4E5B9) & MASK64
    z ^= z >> 27
    z = (z * 0x94D049BB133111EB) & MASK64
    z ^= z >> 31
    return z


def _mix64_inplace(z: np.ndarray, t: np.ndarray) -> None:
    np.right_shift(z, np.uint64(30), out=t)
    z ^= t
    z *= np.uint64(0xBF58476D1CE4E5B9)
    np.right_shift(z, np.uint64(27), out=t)
    z ^= t
    z *= np.uint64(0x94D049BB133111EB)
    np.right_shift(z, np.uint64(31), out=t)
    z ^= t


class _Feistel:
    """Keyed bijection of [0, n): the same network as the library's host/device generators."""

    def __init__(self, n: int, seed: int):
        k = 2
        while k < 64 and (1 << k) < n:
            k += 1
        self.n = n
        self.lo_bits, self.hi_bits = k // 2, k - k // 2
        self.lo_mask = np.uint64((1 << self.lo_bits) - 1)
        self.hi_mask = np.uint64((1 << self.hi_bits) - 1)
        s, self.keys = seed & MASK64, []
        for _ in range(6):
            s = (s + _GOLDEN) & MASK64
            self.keys.append(np.uint64(_mix64_int(s)))

    def _pass(self, x: np.ndarray) -> np.ndarray:
        lo = x & self.lo_mask
        hi = (x >> np.uint64(self.lo_bits)) & self.hi_mask
        f, t = np.empty_like(lo), np.empty_like(lo)
        for r in range(6):
            src, dst, mask = (lo, hi, self.hi_mask) if r % 2 == 0 else (hi, lo, self.lo_mask)
            np.bitwise_xor(src, self.keys[r], out=f)
            _mix64_inplace(f, t)
            f &= mask
            dst ^= f
        hi <<= np.uint64(self.lo_bits)
        hi |= lo
        return hi

    def perm(self, idx: np.ndarray) -> np.ndarray:
        if self.n <= 1:
            return np.zeros_like(idx)
        y = self._pass(idx)
        out = y >= np.uint64(self.n)
        while out.any():  # cycle walking
            sel = np.nonzero(out)[0]
            y[sel] = self._pass(y[sel])
            out[sel] = y[sel] >= np.uint64(self.n)
        return y


def gen_fast_into(R: np.ndarray, S: np.ndarray, seed: int = 12345, payload: bool = False, dup: int = 1,
                  threads: int | None = None, chunk: int = 1 << 16) -> None:
    """Fill R (nR x 2 uint64) and S (nS x 2 uint64) - np.memmap views of .bin files included - with the
    bytes hj_gen_fast_host writes for (nR, nS, seed, payload, dup). Chunks run on a thread pool (numpy
    releases the GIL inside its loops)."""
    import concurrent.futures

    nR, nS = R.shape[0], S.shape[0]
    dup = max(1, int(dup))
    distinct = (nR + dup - 1) // dup
    payload = bool(payload) or dup > 1
    fr = _Feistel(nR, (seed ^ 0x5245) & MASK64)
    fs = _Feistel(nS if nS else 1, (seed ^ 0x53 ^ 0x7F4A7C159E3779B9) & MASK64)

    def fill(out, f, lo, hi, side_r):
        idx = np.arange(lo, hi, dtype=np.uint64)
        p = f.perm(idx)
        if side_r and distinct == f.n:
            key = p + np.uint64(1)
        else:
            key = p % np.uint64(distinct) + np.uint64(1)
        out[lo:hi, 0] = key
        out[lo:hi, 1] = idx + np.uint64(1) if payload else key

    jobs = [(R, fr, lo, min(nR, lo + chunk), True) for lo in range(0, nR, chunk)]
    jobs += [(S, fs, lo, min(nS, lo + chunk), False) for lo in range(0, nS, chunk)]
    with concurrent.futures.ThreadPoolExecutor(max_workers=threads or os.cpu_count() or 1) as ex:
        for fut in [ex.submit(fill, *j) for j in jobs]:
            fut.result()


def gen_fast(nR: int, nS: int, seed: int = 12345, payload: bool = False, dup: int = 1,
             threads: int | None = None):
    R = np.empty((nR, 2), dtype=np.uint64)
    S = np.empty((nS, 2), dtype=np.uint64)
    gen_fast_into(R, S, seed, payload, dup, threads)
    return R, S


def gen_fast_files(prefix: str, rfile: str, sfile: str, nR: int, nS: int, seed: int = 12345,
                   threads: int | None = None) -> None:
    """Write gen_fast's relations (payload = key) straight into two raw .bin files of 16-byte tuples."""
    R = np.memmap(os.path.join(prefix, rfile), dtype=np.uint64, mode="w+", shape=(nR, 2))
    S = np.memmap(os.path.join(prefix, sfile), dtype=np.uint64, mode="w+", shape=(nS, 2))
    gen_fast_into(R, S, seed, threads=threads)
    R.flush()
    S.flush()
    del R, S


def pkfk_closed_form(nR: int, nS: int) -> tuple[int, int]:
    """PK-FK uniform data with row_id = key and nS a multiple of nR: every probe tuple matches once and
    check_sum = m n (n + 1) mod 2^64 with m = nS / nR (the reference's closed form)."""
    m = nS // nR
    return nS, (m * nR * (nR + 1)) & MASK64


# ------------------------------------------------------------------------------------------------
# C oracle
# ------------------------------------------------------------------------------------------------
_lib = None


def build() -> None:
    subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True, capture_output=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        vp, sz, u64p = ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64)
        L.hjo_join.argtypes = [ctypes.c_int, vp, sz, vp, sz, u64p, u64p]
        L.hjo_join.restype = ctypes.c_int
        L.hjo_phj_literal.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, sz, vp, sz, u64p, u64p]
        L.hjo_phj_literal.restype = ctypes.c_int
        L.hjo_join_dense.argtypes = [ctypes.c_int, vp, sz, vp, sz, ctypes.c_uint64, u64p, u64p]
        L.hjo_join_dense.restype = ctypes.c_int
        _lib = L
    return _lib


def _arr(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    assert a.ndim == 2 and a.shape[1] == 2
    return a


def join(mode_or_algo, R: np.ndarray, S: np.ndarray) -> tuple[int, int]:
    """(matched_cnt, check_sum) from the definition of the join (hj_oracle.c hjo_join)."""
    mode = MODE_OF_ALGO[mode_or_algo] if isinstance(mode_or_algo, str) else mode_or_algo
    R, S = _arr(R), _arr(S)
    c, s = ctypes.c_uint64(), ctypes.c_uint64()
    rc = lib().hjo_join(mode, R.ctypes.data, R.shape[0], S.ctypes.data, S.shape[0], ctypes.byref(c),
                        ctypes.byref(s))
    assert rc == 0, rc
    return c.value, s.value


def join_pairs(mode_or_algo, R: np.ndarray, S: np.ndarray) -> np.ndarray:
    """The (r.row_id, s.row_id) pairs of a join from its definition, sorted (n, 2) uint64: what the
    reference's ptr_* joins write into their materialisation buffer (src/algo/ptr_phj.c:689-783, one
    pair per match; lp joins: one pair per probe tuple with a match, the first build tuple in input
    order, key 0 never matching for phj_radix_lp)."""
    mode = MODE_OF_ALGO[mode_or_algo[4:] if isinstance(mode_or_algo, str) and mode_or_algo.startswith("ptr_")
                        else mode_or_algo] if isinstance(mode_or_algo, str) else mode_or_algo
    R, S = _arr(R), _arr(S)
    rpos = np.arange(R.shape[0])
    if mode == FIRST:
        rpos = rpos[R[:, 0] != 0]  # key 0 is an empty slot of lp_join (src/algo/phj.c:614)
    rk = R[rpos, 0]
    order = np.argsort(rk, kind="stable")  # equal keys stay in input order
    rks, rps = rk[order], rpos[order]
    sk = S[:, 0]
    lo = np.searchsorted(rks, sk, "left")
    hi = np.searchsorted(rks, sk, "right")
    if mode == ALL:
        cnt = hi - lo
        s_idx = np.repeat(np.arange(S.shape[0]), cnt)
        start = np.repeat(lo, cnt)
        within = np.arange(s_idx.shape[0]) - np.repeat(np.cumsum(cnt) - cnt, cnt)
        r_idx = rps[start + within]
    else:
        m = hi > lo
        s_idx = np.nonzero(m)[0]
        r_idx = rps[lo[m]]
    out = np.stack([R[r_idx, 1], S[s_idx, 1]], axis=1).astype(np.uint64)
    return out[np.lexsort((out[:, 1], out[:, 0]))]


def join_dense(mode_or_algo, R: np.ndarray, S: np.ndarray, max_key: int) -> tuple[int, int]:
    mode = MODE_OF_ALGO[mode_or_algo] if isinstance(mode_or_algo, str) else mode_or_algo
    R, S = _arr(R), _arr(S)
    c, s = ctypes.c_uint64(), ctypes.c_uint64()
    rc = lib().hjo_join_dense(mode, R.ctypes.data, R.shape[0], S.ctypes.data, S.shape[0], max_key,
                              ctypes.byref(c), ctypes.byref(s))
    assert rc == 0, rc
    return c.value, s.value


def phj_literal(bits: int, passes: int, lp: bool, R: np.ndarray, S: np.ndarray) -> tuple[int, int, int]:
    """Step-by-step restatement of the reference's radix join; returns (cnt, sum, rc)."""
    R, S = _arr(R), _arr(S)
    c, s = ctypes.c_uint64(), ctypes.c_uint64()
    rc = lib().hjo_phj_literal(bits, passes, 1 if lp else 0, R.ctypes.data, R.shape[0], S.ctypes.data,
                               S.shape[0], ctypes.byref(c), ctypes.byref(s))
    return c.value, s.value, rc


# ------------------------------------------------------------------------------------------------
# The reference itself (oracle/_ref, built from its sources by oracle/Makefile)
# ------------------------------------------------------------------------------------------------
# Where the reference's sources are: $HJ_REFERENCE_ROOT, else the REF default of oracle/Makefile (the
# recipe that compiles them). Machines that only run the prebuilt binaries have no sources.
def _reference_root() -> pathlib.Path | None:
    env = os.environ.get("HJ_REFERENCE_ROOT")
    if env:
        return pathlib.Path(env)
    m = re.search(r"^REF \?= *(\S+)", (HERE / "Makefile").read_text(), re.M)
    return pathlib.Path(m.group(1)) if m else None


_REF_ROOT = _reference_root()
REF_SOURCES = _REF_ROOT / "src" if _REF_ROOT else None


def ref_sources_present() -> bool:
    return REF_SOURCES is not None and (REF_SOURCES / "algo" / "phj.c").exists()


def ref_available(passes: int = 2) -> bool:
    return (REF_DIR / f"hjref_p{passes}").exists()


def ref_build() -> bool:
    if not ref_sources_present():
        return ref_available(1) and ref_available(2)
    env = dict(os.environ)
    if _REF_ROOT is not None:
        env["REF"] = str(_REF_ROOT)
    out = subprocess.run(["make", "-C", str(HERE), "ref"], capture_output=True, text=True, env=env)
    return out.returncode == 0


def ref_gen(kind: str, nR: int, nS: int, factor: float = 1.05, seed: int = 12345):
    """Relations written by the reference's own generator functions (src/gen.c)."""
    with tempfile.TemporaryDirectory() as d:
        cmd = [str(REF_DIR / "hjref_p2"), f"--gen={kind}", f"--prefix={d}", f"--nr={nR}", f"--ns={nS}",
               f"--seed={seed}", f"--factor={factor}"]
        subprocess.run(cmd, check=True, capture_output=True, timeout=600)
        if kind == "zipf":
            path = pathlib.Path(d) / "zipfian" / f"fk_{factor:.3f}_AS.bin"
            return np.fromfile(path, dtype=np.uint64).reshape(-1, 2)
        prefix = "dup" if kind == "dup" else "pk"
        R = np.fromfile(pathlib.Path(d) / "gen" / f"{prefix}_R.bin", dtype=np.uint64).reshape(-1, 2)
        S = np.fromfile(pathlib.Path(d) / "gen" / "fk_S.bin", dtype=np.uint64).reshape(-1, 2)
        return R, S


_REF_LINE = re.compile(r"matched_cnt: (\d+)\s+check_sum: (\d+)")
_TRIAL_LINE = re.compile(r"hjref_trial: (\d+) buildpart: ([\d.eE+-]+) probejoin: ([\d.eE+-]+) total: ([\d.eE+-]+)")


def ref_run_files(algo: str, prefix: str, rfile: str, sfile: str, nR: int, nS: int, bits: int = 14,
                  passes: int = 2, threads: int | None = None, trials: int = 1, timeout: float = 900,
                  bits1: int = 11):
    """Run the reference's join on .bin files; returns [(cnt, sum, buildpart, probejoin, total)].
    bits1 is NUM_RADIX_BITS_PASS1 of the phj_asymm_radix_* joins."""
    threads = threads or os.cpu_count() or 1
    cmd = [str(REF_DIR / f"hjref_p{passes}"), f"--algo={algo}", f"--prefix={prefix}", f"--r={rfile}",
           f"--s={sfile}", f"--nr={nR}", f"--ns={nS}", f"--bits={bits}", f"--threads={threads}",
           f"--trials={trials}", f"--bits1={bits1}"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if out.returncode != 0:
        raise RuntimeError(f"reference run failed ({out.returncode}): {out.stderr[-2000:]}")
    res = [(int(a), int(b)) for a, b in _REF_LINE.findall(out.stdout)]
    tim = [(float(b), float(c), float(d)) for _, b, c, d in _TRIAL_LINE.findall(out.stdout)]
    return [r + t for r, t in zip(res, tim)]


def ref_join(algo: str, R: np.ndarray, S: np.ndarray, bits: int = 14, passes: int = 2,
             threads: int | None = None, bits1: int = 11) -> tuple[int, int]:
    """(matched_cnt, check_sum) printed by the reference's own join on these relations."""
    with tempfile.TemporaryDirectory() as d:
        _arr(R).tofile(os.path.join(d, "r.bin"))
        _arr(S).tofile(os.path.join(d, "s.bin"))
        runs = ref_run_files(algo, d, "r.bin", "s.bin", R.shape[0], S.shape[0], bits, passes, threads,
                             bits1=bits1)
        return runs[0][0], runs[0][1]


# ------------------------------------------------------------------------------------------------
# Sharded joins: the owner of a key (the library's hj_shard_route) and a host routing of a relation
# ------------------------------------------------------------------------------------------------
def shard_of(keys: np.ndarray, nshards: int) -> np.ndarray:
    """owner = mulhi(mix64(key ^ 0x5ca1ab1e5eed0001), nshards), mix64 = splitmix64's output mix."""
    z = np.asarray(keys, dtype=np.uint64) ^ np.uint64(0x5CA1AB1E5EED0001)
    t = np.empty_like(z)
    _mix64_inplace(z, t)
    hi, lo = z >> np.uint64(32), z & np.uint64(0xFFFFFFFF)
    n = np.uint64(nshards)
    return ((hi * n + ((lo * n) >> np.uint64(32))) >> np.uint64(32)).astype(np.int64)


def shard_route(T: np.ndarray, nshards: int):
    """Stable grouping of the tuples of T (n x 2) by owner: (routed tuples, tuples per owner)."""
    own = shard_of(T[:, 0], nshards)
    order = np.argsort(own, kind="stable")
    return T[order], np.bincount(own, minlength=nshards).astype(np.int64)
