"""CPU check of segment mode's index arithmetic (the design of seg_pass1_kernel in
hashjoin-scm_b200/csrc/hj_partition.cu, restated tile by tile in numpy): with pass-1 CTAs taking work
items in an interleaved order, every store lands inside the segment storage, no slot is written twice,
segment ids stay below the bound that phj_carve reserves (floor(n / 2048) + 2 * CTAs * F1 + 32 * CTAs),
and walking each (CTA, relation, digit) chain for its histogram count returns exactly that CTA's tuples
of that digit. Segments hold 2048 tuples, or 4096 8-byte words when pass 1 stores words (the same 32 KB;
pass 2 then reads one segment per 4096-word tile). No GPU is used."""
import numpy as np
import pytest

T = 2048          # tuples per pass-1 tile (and per segment of tuples)
SLAB = 32         # segment ids a CTA takes from the global counter at once
NONE = 0xFFFFFFFF


def emulate(nR, nS, bits, F1, G, it_tiles, seed, skew=False, segw=T):
    rng = np.random.default_rng(seed)
    hi = 50 if skew else 1 << 40
    rels = [rng.integers(1, hi, nR, dtype=np.uint64), rng.integers(1, hi, nS, dtype=np.uint64)]
    nbins = 1 << bits
    tiles = [-(-nR // T), -(-nS // T)]
    itemsR = -(-tiles[0] // it_tiles)
    items = itemsR + -(-tiles[1] // it_tiles)
    max_segs = (nR + nS) // T + 2 * G * F1 + G * SLAB  # reserved for 2048-tuple segments
    cap = max_segs * segw
    out = np.full(cap, -1, dtype=np.int64)
    seg_head = np.full((2 * G, F1), -1, dtype=np.int64)
    seg_next = np.full(max_segs, -1, dtype=np.int64)
    hist = np.zeros((2 * G, nbins), dtype=np.int64)
    alloc = 0
    st = [dict(cur=[NONE] * F1, fill=[0] * F1, lo=0, rem=0, rel=0, item=None, tn=0, te=0) for _ in range(G)]
    next_item = 0
    active = list(range(G))
    turn = 0
    while active:
        c = active[turn % len(active)]
        s = st[c]
        while s["item"] is None or s["tn"] >= s["te"]:
            it = next_item
            next_item += 1
            if it >= items:
                s["item"] = None
                break
            rel = int(it >= itemsR)
            k = it - itemsR if rel else it
            s["item"], s["tn"], s["te"] = it, k * it_tiles, min(k * it_tiles + it_tiles, tiles[rel])
        if s["item"] is None:
            active.remove(c)
            continue
        turn += 1
        rel = int(s["item"] >= itemsR)
        lo = s["tn"] * T
        n = len(rels[rel])
        cnt = min(T, n - lo)
        s["tn"] += 1
        if rel != s["rel"]:  # R tiles come first: start S's chains
            s["cur"], s["fill"], s["rel"] = [NONE] * F1, [0] * F1, rel
        keys = rels[rel][lo:lo + cnt]
        d = (keys & np.uint64(F1 - 1)).astype(np.int64)
        np.add.at(hist[rel * G + c], (keys & np.uint64(nbins - 1)).astype(np.int64), 1)
        h = np.bincount(d, minlength=F1)
        order = np.argsort(d, kind="stable")  # staged tile, sorted by digit
        ex = np.concatenate([[0], np.cumsum(h)[:-1]])
        need = [int(h[x] > 0 and (s["cur"][x] == NONE or s["fill"][x] + h[x] > segw)) for x in range(F1)]
        ntot = sum(need)
        old_lo, old_rem, nb = s["lo"], s["rem"], 0
        if ntot:
            if ntot <= s["rem"]:
                s["lo"] += ntot
                s["rem"] -= ntot
            else:
                deficit = ntot - s["rem"]
                take = max(deficit, SLAB)
                nb, alloc = alloc, alloc + take
                s["lo"], s["rem"] = nb + deficit, take - deficit
        e = 0
        base, jump, split = [0] * F1, [0] * F1, [0] * F1
        row = rel * G + c
        for x in range(F1):
            hh, e0 = int(h[x]), int(ex[x])
            if not hh:
                continue
            sc, fill = s["cur"][x], s["fill"][x]
            if sc != NONE and fill + hh <= segw:
                base[x], split[x] = sc * segw + fill - e0, e0 + hh
                s["fill"][x] = fill + hh
                continue
            sid = old_lo + e if e < old_rem else nb + (e - old_rem)
            e += 1
            assert sid < max_segs, "segment id beyond the reserved storage"
            if sc == NONE:
                seg_head[row, x] = sid
                base[x], split[x] = sid * segw - e0, e0 + hh
                s["fill"][x] = hh
            else:
                seg_next[sc] = sid
                base[x], jump[x], split[x] = sc * segw + fill - e0, sid - sc - 1, e0 + (segw - fill)
                s["fill"][x] = hh - (segw - fill)
            s["cur"][x] = sid
        for j in range(cnt):
            src = int(order[j])
            x = int(d[src])
            dst = base[x] + j + (0 if j < split[x] else jump[x] * segw)
            assert 0 <= dst < cap
            assert out[dst] == -1, "slot written twice"
            out[dst] = (rel << 40) | (lo + src)
    assert alloc <= max_segs
    seen = np.zeros(nR + nS, dtype=np.int64)
    for row in range(2 * G):
        rel = row // G
        for x in range(F1):
            want = int(hist[row, x::F1].sum())  # pass-2 unit size: the row's bins with pass-1 digit x
            sid, done = int(seg_head[row, x]), 0
            while done < want:
                assert 0 <= sid < max_segs
                k = min(segw, want - done)
                vals = out[sid * segw:sid * segw + k]
                assert (vals >= 0).all(), "chain reaches an unwritten slot"
                r = vals >> 40
                idx = vals & ((1 << 40) - 1)
                assert (r == rel).all()
                assert ((rels[rel][idx] & np.uint64(F1 - 1)).astype(np.int64) == x).all()
                np.add.at(seen, idx + (nR if rel else 0), 1)
                done += k
                if done < want:
                    sid = int(seg_next[sid])
    assert (seen == 1).all(), "a tuple is missing or repeated"
    return alloc, max_segs


@pytest.mark.parametrize("segw", [2048, 4096])
@pytest.mark.parametrize("nR,nS,bits,F1,G,it_tiles,seed,skew", [
    (5000, 20000, 4, 4, 3, 1, 1, False),
    (100_000, 300_001, 6, 8, 5, 2, 2, False),
    (70_000, 250_000, 6, 8, 4, 3, 3, True),      # few keys: whole tiles of one digit, long chains
    (1, 1, 4, 4, 3, 1, 4, False),
    (2048 * 7, 2048 * 9 + 5, 8, 16, 2, 16, 5, True),
    (300_000, 10, 10, 32, 7, 4, 6, False),       # almost only R; CTAs without S tiles
])
def test_segment_chains(nR, nS, bits, F1, G, it_tiles, seed, skew, segw):
    used, bound = emulate(nR, nS, bits, F1, G, it_tiles, seed, skew, segw)
    assert used <= bound
