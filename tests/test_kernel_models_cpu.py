"""The arithmetic the codec kernels use in place of the reference's
sequential loops, restated in numpy-free Python and checked against the
oracle on the CPU (the kernels themselves are checked on the GPU by the
parity tests):

* RLE1 (csrc/rle1.cu): which of 16 consecutive bytes emit output, from the
  bit mask of run starts and the position of the first byte in its chunk
  of `cut`; and a tile's output count for the bytes that continue a run
  from an earlier tile, in closed form.
* RLE2 (csrc/rle2.cu): the RUNA/RUNB digits of a zero run of length n are
  the bits of n + 1 below its top bit.
* MTF (csrc/mtf.cu): move-to-front indices from occurrences: a 128-bit mask
  of last occurrences per lane chunk and, for a first-seen symbol, its rank
  in the chunk's starting list less the seen symbols ranked below it; the
  starting lists chained chunk by chunk as rank tables.
"""
import random

import numpy as np
import pytest

import oracle


def _popc(x: int) -> int:
    return bin(x).count("1")


# ------------------------------------------------------------------- RLE1
def _emit_loop(sm, q0, nv, cut, carry):
    """The reference's walk: position q in the run's chunk, reset at starts."""
    e = e3 = 0
    q, on = q0, carry
    for k in range(nv):
        if (sm >> k) & 1:
            q, on = 0, True
        if on and q <= 3:
            e |= 1 << k
        if on and q == 3:
            e3 |= 1 << k
        q = 0 if q + 1 == cut else q + 1
    return e, e3


def _emit_masks(sm, q0, nv, cut, carry):
    """rle1_emit_masks: chunk starts spread over the next 3 bytes."""
    s4 = sm << 4
    if carry:
        if q0 <= 3:
            s4 |= 1 << (4 - q0)
        else:
            pw = cut - q0
            if pw < 16 and (sm & ((1 << pw) - 1)) == 0:
                s4 |= 1 << (pw + 4)
    nvm = (1 << nv) - 1
    e = ((s4 | (s4 << 1) | (s4 << 2) | (s4 << 3)) >> 4) & nvm
    e3 = (((s4 << 3) & ~(s4 << 2) & ~(s4 << 1) & ~s4) >> 4) & nvm
    if not carry:
        keep = ~((sm & -sm) - 1) if sm else 0
        e &= keep
        e3 &= keep
    return e & 0xFFFF, e3 & 0xFFFF


def test_rle1_emit_masks_match_the_position_walk():
    rng = random.Random(5)
    for _ in range(20000):
        cut = rng.choice([255, 259])
        nv = rng.choice([16, 16, rng.randint(0, 16)])
        sm = rng.getrandbits(16) & rng.choice([0, 0xFFFF, rng.getrandbits(16), 1 << rng.randrange(16)])
        q0 = rng.choice([0, 1, 2, 3, 4, rng.randrange(cut), cut - 1, cut - 15, cut - 16])
        carry = rng.random() < 0.8
        assert _emit_masks(sm, q0, nv, cut, carry) == _emit_loop(sm, q0, nv, cut, carry)


def _rle1_out_upto(n, cut):
    f, r = divmod(n, cut)
    return 5 * f + (r if r < 4 else 5)


@pytest.mark.parametrize("cut", [259, 255])
def test_rle1_tile_counts_in_closed_form_sum_to_the_oracle_length(cut):
    rng = random.Random(3 + cut)
    for _ in range(60):
        n = rng.randint(1, 20000)
        parts, tot = [], 0
        while tot < n:
            k = rng.choice([1, 1, 2, 3, 4, 5, rng.randint(1, 3000)])
            parts.append(np.full(k, rng.randrange(4), np.uint8))
            tot += k
        data = np.concatenate(parts)[:n]
        starts = [i for i in range(n) if i == 0 or data[i] != data[i - 1]]
        tile = rng.choice([16, 100, 4096])
        total, carry = 0, -1
        for st in range(0, n, tile):
            ln = min(tile, n - st)
            ts = [s for s in starts if st <= s < st + ln]
            # the tile's own count: from its first run start on
            own, q, on = 0, 0, False
            for x in range(st, st + ln):
                if ts and x in ts:
                    q, on = 0, True
                if on:
                    own += 1 if q < 3 else (2 if q == 3 else 0)
                q = 0 if q + 1 == cut else q + 1
            pre = (ts[0] if ts else st + ln) - st
            j0 = st - carry
            total += own + (_rle1_out_upto(j0 + pre, cut) - _rle1_out_upto(j0, cut) if pre else 0)
            if ts:
                carry = ts[-1]
        assert total == oracle.rle1_cut(data, cut).size


# ------------------------------------------------------------------- RLE2
def test_rle2_run_digits_are_the_bits_of_length_plus_one():
    for n in range(1, 20000):
        x, walk = n, []
        for _ in range((n + 1).bit_length() - 1):  # the reference's loop
            x -= 1
            walk.append(x & 1)
            x >>= 1
        assert walk == [((n + 1) >> q) & 1 for q in range((n + 1).bit_length() - 1)]


# -------------------------------------------------------------------- MTF
def _mtf_from_occurrences(tile, start_list, sub=128):
    ranks = [dict() for _ in range(32)]
    for j, c in enumerate(start_list):
        ranks[0][c] = j
    chunks = [tile[l * sub:(l + 1) * sub] for l in range(32)]
    rec, dist = [], []
    for ch in chunks:  # recency ranks: backward scan of each chunk
        r, k = {}, 0
        for c in reversed(ch):
            if c not in r:
                r[c], k = k, k + 1
        rec.append(r)
        dist.append(k)
    for k in range(1, 32):  # starting lists, chunk by chunk
        seen = sorted(ranks[k - 1][c] for c in start_list if c in rec[k - 1])
        for c in start_list:
            r = ranks[k - 1][c]
            below = sum(1 for x in seen if x < r)
            ranks[k][c] = rec[k - 1][c] if c in rec[k - 1] else dist[k - 1] + r - below
    out = []
    for l, ch in enumerate(chunks):
        last, L, S, dc = {}, 0, 0, 0
        for i, c in enumerate(ch):
            p = last.get(c)
            last[c] = i
            if p is not None:
                idx = dc - _popc(L & ((2 << p) - 1))
                L ^= 1 << p
            else:
                r = ranks[l][c]
                idx = dc + r - _popc(S & ((1 << r) - 1))
                S |= 1 << r
                dc += 1
            L |= 1 << i
            out.append(idx)
    return out


@pytest.mark.parametrize("alphabet", [1, 3, 50, 256])
def test_mtf_from_occurrences_matches_the_oracle(alphabet):
    rng = np.random.default_rng(alphabet)
    symbols = rng.permutation(256)[:alphabet].astype(np.uint8)
    for n in (4096, 1000, 129):
        w = rng.random(alphabet) ** 8
        tile = symbols[rng.choice(alphabet, n, p=w / w.sum())]
        sa = ((np.arange(n) + 1) % n).astype(np.int32)  # the last column is the tile itself
        ref, _, _, _ = oracle.mtf(tile, sa)
        start = sorted(int(c) for c in set(tile.tolist()))  # the oracle's start list
        assert _mtf_from_occurrences([int(c) for c in tile], start) == ref.tolist()
