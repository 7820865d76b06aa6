"""CPU oracle of the bzip2gpu compression path -- TEST INFRASTRUCTURE ONLY.

ctypes view of oracle/bz2_oracle.c (built to oracle/_build/liboracle.so by
`make -C oracle`).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg use it, as the checker; the product library never does.

Also loads, when present, oracle/_ref/libref_testoracles.so: the reference's
own CPU test oracles compiled from the reference tree (`make -C oracle ref`).
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref_testoracles.so"
_lib = None
_ref = None
G, A = 6, 258

_vp, _i = ctypes.c_void_p, ctypes.c_int


class BlockInfo(ctypes.Structure):
    _fields_ = [("n", _i), ("m", _i), ("s", _i), ("n_in_use", _i), ("orig_ptr", _i),
                ("n_groups", _i), ("n_selectors", _i), ("crc", ctypes.c_uint32),
                ("payload_bits", ctypes.c_int64), ("header_bits", ctypes.c_int64),
                ("active_sum", ctypes.c_int64), ("present", ctypes.c_uint8 * 256),
                ("len", (ctypes.c_uint8 * A) * G), ("code", (ctypes.c_int32 * A) * G)]


def build() -> Path:
    if not LIB.exists() or LIB.stat().st_mtime < max(
            (HERE / f).stat().st_mtime
            for f in ("bz2_oracle.c", "bz2_oracle.h", "gen_oracle.c", "blocks.c")):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        L.orc_crc32.restype = ctypes.c_uint32
        L.orc_crc32.argtypes = [_vp, ctypes.c_size_t]
        L.orc_rle1.argtypes = [_vp, _i, _vp]
        L.orc_bwt.argtypes = [_vp, _i, _vp]
        L.orc_bwt_stats.argtypes = [_vp, _i, _vp, ctypes.POINTER(ctypes.c_int64),
                                    ctypes.POINTER(_i)]
        L.orc_mtf.argtypes = [_vp, _vp, _i, _vp, ctypes.POINTER(_i), _vp]
        L.orc_symbols_table.argtypes = [_vp, _i, _vp]
        L.orc_rle2.argtypes = [_vp, _i, _i, _vp]
        L.orc_code_lengths.argtypes = [_vp, _vp, _i, _i]
        L.orc_huffman_build.argtypes = [_vp, _i, _i, _vp, _vp, _vp, ctypes.POINTER(_i)]
        L.orc_huffman_build_passes.argtypes = [_vp, _i, _i, _i, _vp, _vp, _vp, ctypes.POINTER(_i)]
        L.orc_encode.restype = ctypes.c_int64
        L.orc_encode.argtypes = [_vp, _i, _vp, _vp, _vp, _vp]
        L.orc_selector_mtf.argtypes = [_vp, _i, _i, _vp]
        L.orc_huffman_refine.argtypes = [_vp, _i, _i, _vp, _i, _vp, _vp, _vp]
        L.orc_huffman_learned.argtypes = [_vp, _i, _i, _vp, _vp, _vp, _vp, ctypes.POINTER(_i),
                                          ctypes.POINTER(_i)]
        L.orc_coded_bits.restype = ctypes.c_int64
        L.orc_coded_bits.argtypes = [_vp, _i, _vp, _i, _i, _vp]
        L.orc_compress_block.argtypes = [_vp, _i, ctypes.POINTER(BlockInfo), _vp, _vp, _vp, _vp,
                                         _vp]
        L.orc_compress.restype = ctypes.c_int64
        L.orc_compress.argtypes = [_vp, ctypes.c_int64, _i, _i, _vp, ctypes.c_int64, _i]
        L.orc_compress_part.restype = ctypes.c_int64
        L.orc_compress_part.argtypes = [_vp, ctypes.c_int64, _i, _vp, ctypes.c_int64, _i,
                                        ctypes.POINTER(ctypes.c_int64),
                                        ctypes.POINTER(ctypes.c_uint32)]
        L.orc_assemble.restype = ctypes.c_int64
        L.orc_assemble.argtypes = [_i, _vp, _vp, _vp, _vp, _i, _vp, ctypes.c_int64]
        L.orc_rle1_cut.argtypes = [_vp, _i, _vp, _i]
        L.orc_bzip2_split.restype = ctypes.c_int64
        L.orc_bzip2_split.argtypes = [_vp, ctypes.c_int64, _i, _vp, ctypes.c_int64]
        L.orc_compress_bound.restype = ctypes.c_int64
        L.orc_compress_bound.argtypes = [ctypes.c_int64, _i]
        L.orc_gen_markov.argtypes = [ctypes.c_uint64, _vp, _i, ctypes.c_double, ctypes.c_double,
                                     _i, _i, _vp, ctypes.c_int64, _i]
        L.orc_gen_uniform.argtypes = [ctypes.c_uint64, _vp, ctypes.c_int64, _i]
        L.orc_scan_magic.restype = ctypes.c_int64
        L.orc_scan_magic.argtypes = [_vp, ctypes.c_int64, _i, _vp, ctypes.c_int64, _i]
        L.orc_rewrap_block.restype = ctypes.c_int64
        L.orc_rewrap_block.argtypes = [_vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, _i,
                                       _vp]
        _lib = L
    return _lib


def ref_lib():
    """The reference's own CPU test oracles, or None if not built here."""
    global _ref
    if _ref is None and REF_LIB.exists():
        R = ctypes.CDLL(str(REF_LIB))
        R.ref_rle1.argtypes = [_vp, _i, _vp]
        R.ref_bwt.argtypes = [_vp, _i, _vp]
        R.ref_mtf_plain.argtypes = [_vp, _i, _vp]
        R.ref_rle2.argtypes = [_vp, _i, _i, _vp]
        _ref = R
    return _ref


def _u8(a) -> np.ndarray:
    return np.ascontiguousarray(np.frombuffer(a, np.uint8) if isinstance(a, (bytes, bytearray))
                                else a, dtype=np.uint8).reshape(-1)


def crc32(data) -> int:
    a = _u8(data)
    return lib().orc_crc32(a.ctypes.data, a.size)


def rle1(data) -> np.ndarray:
    a = _u8(data)
    out = np.zeros(a.size + a.size // 4 + 8, np.uint8)
    m = lib().orc_rle1(a.ctypes.data, a.size, out.ctypes.data)
    return out[:m].copy()


def bwt(data) -> np.ndarray:
    a = _u8(data)
    sa = np.zeros(max(a.size, 1), np.int32)
    lib().orc_bwt(a.ctypes.data, a.size, sa.ctypes.data)
    return sa[: a.size].copy()


def bwt_stats(data):
    a = _u8(data)
    sa = np.zeros(max(a.size, 1), np.int32)
    act = ctypes.c_int64()
    rounds = _i()
    lib().orc_bwt_stats(a.ctypes.data, a.size, sa.ctypes.data, ctypes.byref(act),
                        ctypes.byref(rounds))
    return sa[: a.size].copy(), act.value, rounds.value


def mtf(orig, sa):
    """(mtf values, origPtr, present[256], nInUse)"""
    o = _u8(orig)
    s = np.ascontiguousarray(sa, dtype=np.int32)
    out = np.zeros(max(o.size, 1), np.uint8)
    op = _i(-1)
    pres = np.zeros(256, np.uint8)
    n = lib().orc_mtf(o.ctypes.data, s.ctypes.data, o.size, out.ctypes.data, ctypes.byref(op),
                      pres.ctypes.data)
    return out[: o.size].copy(), op.value, pres, n


def symbols_table(data) -> np.ndarray:
    a = _u8(data)
    t = np.zeros(256, np.uint8)
    n = lib().orc_symbols_table(a.ctypes.data, a.size, t.ctypes.data)
    return t[:n].copy()


def rle2(mtf_vals, table_size: int) -> np.ndarray:
    a = _u8(mtf_vals)
    out = np.zeros(a.size + 2, np.uint16)
    s = lib().orc_rle2(a.ctypes.data, a.size, table_size, out.ctypes.data)
    return out[:s].copy()


def code_lengths(freq, alpha_size: int, max_len: int = 17) -> np.ndarray:
    f = np.ascontiguousarray(freq, dtype=np.int32)
    ln = np.zeros(A, np.uint8)
    lib().orc_code_lengths(f.ctypes.data, ln.ctypes.data, alpha_size, max_len)
    return ln[:alpha_size].copy()


def huffman_build(syms, n_in_use: int, passes: int = 4):
    """(len[6,258], code[6,258], selectors, n_groups) of the plain selector
    with `passes` selection passes (the reference's 4)."""
    s = np.ascontiguousarray(syms, dtype=np.uint16)
    ln = np.zeros((G, A), np.uint8)
    code = np.zeros((G, A), np.int32)
    sel = np.zeros(s.size // 50 + 2, np.uint8)
    ng = _i()
    nsel = lib().orc_huffman_build_passes(s.ctypes.data, s.size, n_in_use, passes, ln.ctypes.data,
                                          code.ctypes.data, sel.ctypes.data, ctypes.byref(ng))
    return ln, code, sel[:nsel].copy(), ng.value


def encode(syms, selectors, len_tab, code_tab):
    s = np.ascontiguousarray(syms, dtype=np.uint16)
    sel = np.ascontiguousarray(selectors, dtype=np.uint8)
    lt = np.ascontiguousarray(len_tab, dtype=np.uint8)
    ct = np.ascontiguousarray(code_tab, dtype=np.int32)
    words = np.zeros(s.size * 17 // 32 + 2, np.uint32)
    bits = lib().orc_encode(s.ctypes.data, s.size, sel.ctypes.data, lt.ctypes.data,
                            ct.ctypes.data, words.ctypes.data)
    return words[: (bits + 31) // 32].copy(), bits


def huffman_refine(syms, n_in_use: int, sel_in, n_refine: int = 1):
    """The learned form after its first assignment sel_in (six tables):
    (len[6,258], code[6,258], selectors)."""
    s = np.ascontiguousarray(syms, dtype=np.uint16)
    si = np.ascontiguousarray(sel_in, dtype=np.uint8)
    ln = np.zeros((G, A), np.uint8)
    code = np.zeros((G, A), np.int32)
    sel = np.zeros(s.size // 50 + 2, np.uint8)
    nsel = lib().orc_huffman_refine(s.ctypes.data, s.size, n_in_use, si.ctypes.data, n_refine,
                                    ln.ctypes.data, code.ctypes.data, sel.ctypes.data)
    return ln, code, sel[:nsel].copy()


def huffman_learned(syms, n_in_use: int, sel_mlp):
    """The learned form given the MLP's choices: (len, code, selectors,
    n_groups, fell_back)."""
    s = np.ascontiguousarray(syms, dtype=np.uint16)
    sm = np.ascontiguousarray(sel_mlp, dtype=np.uint8)
    ln = np.zeros((G, A), np.uint8)
    code = np.zeros((G, A), np.int32)
    sel = np.zeros(s.size // 50 + 2, np.uint8)
    ng, fb = _i(), _i()
    nsel = lib().orc_huffman_learned(s.ctypes.data, s.size, n_in_use, sm.ctypes.data,
                                     ln.ctypes.data, code.ctypes.data, sel.ctypes.data,
                                     ctypes.byref(ng), ctypes.byref(fb))
    return ln, code, sel[:nsel].copy(), ng.value, bool(fb.value)


def coded_bits(syms, selectors, n_groups: int, n_in_use: int, len_tab) -> int:
    """Selection-dependent bits of a block (payload, selector MTF, tables)."""
    s = np.ascontiguousarray(syms, dtype=np.uint16)
    sel = np.ascontiguousarray(selectors, dtype=np.uint8)
    lt = np.ascontiguousarray(len_tab, dtype=np.uint8)
    return lib().orc_coded_bits(s.ctypes.data, s.size, sel.ctypes.data, n_groups, n_in_use,
                                lt.ctypes.data)


def selector_mtf(sel, n_groups: int) -> np.ndarray:
    s = np.ascontiguousarray(sel, dtype=np.uint8)
    out = np.zeros(max(s.size, 1), np.uint8)
    lib().orc_selector_mtf(s.ctypes.data, s.size, n_groups, out.ctypes.data)
    return out[: s.size].copy()


def compress_block(raw):
    """Every stage of one block: dict of arrays and a BlockInfo."""
    a = _u8(raw)
    n = a.size
    cap = n + n // 4 + 8
    r1 = np.zeros(cap, np.uint8)
    sa = np.zeros(cap, np.int32)
    mt = np.zeros(cap, np.uint8)
    r2 = np.zeros(cap + 2, np.uint16)
    sel = np.zeros(cap // 50 + 4, np.uint8)
    info = BlockInfo()
    lib().orc_compress_block(a.ctypes.data, n, ctypes.byref(info), r1.ctypes.data, sa.ctypes.data,
                             mt.ctypes.data, r2.ctypes.data, sel.ctypes.data)
    m, s = info.m, info.s
    return {"rle1": r1[:m].copy(), "sa": sa[:m].copy(), "mtf": mt[:m].copy(),
            "rle2": r2[:s].copy(), "sel": sel[: info.n_selectors].copy(),
            "len": np.array(info.len, np.uint8), "code": np.array(info.code, np.int32)}, info


BZIP2_BLOCKS = -1  # block_bytes value: bzip2 1.0.8's blocks and 255-byte runs


def rle1_cut(data, cut: int) -> np.ndarray:
    a = _u8(data)
    out = np.zeros(a.size + a.size // 4 + 8, np.uint8)
    m = lib().orc_rle1_cut(a.ctypes.data if a.size else None, a.size, out.ctypes.data, cut)
    return out[:m].copy()


def bzip2_split(data, level: int = 9) -> np.ndarray:
    """Block end offsets of bzip2 1.0.8's split of data at `level`."""
    a = _u8(data)
    p = a.ctypes.data if a.size else None
    nb = lib().orc_bzip2_split(p, a.size, level, None, 0)
    ends = np.zeros(max(nb, 1), np.int64)
    lib().orc_bzip2_split(p, a.size, level, ends.ctypes.data, nb)
    return ends[:nb]


def compress(data, level: int = 9, block_bytes: int = 900000, threads: int = 1) -> bytes:
    a = _u8(data)
    cap = lib().orc_compress_bound(a.size, block_bytes)
    out = np.zeros(cap, np.uint8)
    n = lib().orc_compress(a.ctypes.data if a.size else None, a.size, level, block_bytes,
                           out.ctypes.data, cap, threads)
    if n < 0:
        raise RuntimeError("oracle output buffer too small")
    return out[:n].tobytes()


def compress_part(data, block_bytes: int = 900000, threads: int = 1):
    """(part bytes, bits, crc fold, blocks) of the blocks of data."""
    a = _u8(data)
    cap = lib().orc_compress_bound(a.size, block_bytes)
    out = np.zeros(cap + 8, np.uint8)
    bits = ctypes.c_int64()
    fold = ctypes.c_uint32()
    n = lib().orc_compress_part(a.ctypes.data if a.size else None, a.size, block_bytes,
                                out.ctypes.data, cap, threads, ctypes.byref(bits),
                                ctypes.byref(fold))
    if n < 0:
        raise RuntimeError("oracle output buffer too small")
    nb = (a.size + block_bytes - 1) // block_bytes
    return out[:n].copy(), bits.value, fold.value, nb


def assemble(parts, bits, folds, nblocks, level: int = 9) -> bytes:
    k = len(parts)
    arrs = [np.ascontiguousarray(p, dtype=np.uint8) for p in parts]
    ptrs = (ctypes.c_void_p * max(k, 1))(*[p.ctypes.data for p in arrs])
    b = np.ascontiguousarray(bits, dtype=np.int64)
    f = np.ascontiguousarray(folds, dtype=np.uint32)
    nb = np.ascontiguousarray(nblocks, dtype=np.int32)
    cap = int(sum(p.size for p in arrs)) + 64
    out = np.zeros(cap, np.uint8)
    n = lib().orc_assemble(k, ptrs, b.ctypes.data, f.ctypes.data, nb.ctypes.data, level,
                           out.ctypes.data, cap)
    return out[:n].tobytes()



# ------------------------------------------------------------ workload bytes
def _threads(threads):
    import os
    return threads if threads else (os.cpu_count() or 1)


def gen_markov(n: int, seed: int, alphabet, alpha: float, p_run: float, run_min: int,
               run_max: int, threads: int = 0) -> np.ndarray:
    """Order-1 Markov bytes with run starts (definition in gen_oracle.c)."""
    alph = np.ascontiguousarray(alphabet, dtype=np.uint8)
    out = np.empty(n, np.uint8)
    if lib().orc_gen_markov(seed & (2**64 - 1), alph.ctypes.data, alph.size, alpha, p_run,
                            run_min, run_max, out.ctypes.data, n, _threads(threads)) != 0:
        raise ValueError("gen_markov: bad arguments")
    return out


def gen_uniform(n: int, seed: int, threads: int = 0) -> np.ndarray:
    out = np.empty(n, np.uint8)
    if lib().orc_gen_uniform(seed & (2**64 - 1), out.ctypes.data, n, _threads(threads)) != 0:
        raise ValueError("gen_uniform: bad arguments")
    return out


SEGMENT = 64 << 20


def large_stream_segments(n: int, seed: int = 0xB2C4):
    """Parameters of the large Markov stream's 64 MiB segments: (seed,
    alphabet, alpha) per segment, drawn from numpy's PCG64 with `seed`: an
    alphabet size uniform in 2..256 (a random subset of the byte values,
    ascending) and alpha log-uniform in 0.05..5."""
    import math
    rng = np.random.default_rng(seed)
    res = []
    for k in range((n + SEGMENT - 1) // SEGMENT):
        a = int(rng.integers(2, 257))
        alph = np.sort(rng.choice(256, a, replace=False)).astype(np.uint8)
        alpha = float(math.exp(rng.uniform(math.log(0.05), math.log(5.0))))
        res.append((seed * 1000003 + k, alph, alpha))
    return res


def large_stream(n: int, seed: int = 0xB2C4, threads: int = 0) -> np.ndarray:
    """The first n bytes of the large Markov stream (2 % run starts of length
    4..300, parameters redrawn every 64 MiB)."""
    out = np.empty(n, np.uint8)
    for k, (sseed, alph, alpha) in enumerate(large_stream_segments(n, seed)):
        a, b = k * SEGMENT, min(n, (k + 1) * SEGMENT)
        out[a:b] = gen_markov(b - a, sseed, alph, alpha, 0.02, 4, 300, threads)
    return out


def large_stream_sample(n: int, per_segment: int = 1_800_000, seed: int = 0xB2C4,
                        threads: int = 0) -> np.ndarray:
    """A bounded sample of the n-byte large Markov stream that covers every
    one of its parameter redraws: the first `per_segment` bytes of each 64 MiB
    segment (two 900,000-byte blocks by default), back to back.  These are
    the stream's own bytes: a segment's chains do not depend on its length."""
    parts = []
    for k, (sseed, alph, alpha) in enumerate(large_stream_segments(n, seed)):
        seg = min(n, (k + 1) * SEGMENT) - k * SEGMENT
        parts.append(gen_markov(min(per_segment, seg), sseed, alph, alpha, 0.02, 4, 300, threads))
    return np.concatenate(parts) if parts else np.zeros(0, np.uint8)


# ------------------------------------------------- libbz2 decode, in parallel
def _scan(s: np.ndarray, kind: int, threads: int) -> np.ndarray:
    n = lib().orc_scan_magic(s.ctypes.data, s.size, kind, None, 0, threads)
    out = np.zeros(max(n, 1), np.int64)
    lib().orc_scan_magic(s.ctypes.data, s.size, kind, out.ctypes.data, n, threads)
    return out[:n]


def block_bounds(stream, threads: int = 0):
    """(start bit, end bit) of every block of a single .bz2 stream: from each
    block magic to the next one, the last to the end-of-stream magic."""
    s = _u8(stream)
    t = _threads(threads)
    starts = _scan(s, 0, t)
    eos = _scan(s, 1, t)
    if eos.size == 0:
        raise ValueError("no end-of-stream marker")
    end = int(eos[-1])
    starts = starts[starts < end]
    ends = np.append(starts[1:], end)
    return list(zip(starts.tolist(), ends.tolist()))


def rewrap_block(stream, b0: int, b1: int, level: int) -> bytes:
    s = _u8(stream)
    out = np.zeros((b1 - b0) // 8 + 32, np.uint8)
    k = lib().orc_rewrap_block(s.ctypes.data, s.size, b0, b1, level, out.ctypes.data)
    return out[:k].tobytes()


def libbz2_matches(stream, expect, threads: int = 0) -> dict:
    """Decode every block of `stream` with libbz2 (each block re-wrapped as a
    stream of its own, blocks on `threads` threads) and compare the
    concatenated output with `expect` (a host array).  A block magic that is
    really payload bits makes two blocks fail to decode, so the result also
    reports a mismatch then."""
    import bz2
    from concurrent.futures import ThreadPoolExecutor

    s = _u8(stream)
    e = _u8(expect)
    level = int(s[3]) - 48
    bounds = block_bounds(s, threads)

    def dec(bb):
        try:
            return bz2.decompress(rewrap_block(s, bb[0], bb[1], level))
        except (OSError, ValueError):
            return None

    at, ok = 0, True
    with ThreadPoolExecutor(_threads(threads)) as ex:
        for d in ex.map(dec, bounds):
            if d is None or not ok:
                ok = False
                continue
            if d != e[at:at + len(d)].tobytes():
                ok = False
            at += len(d)
    return {"blocks": len(bounds), "bytes": at, "identical": bool(ok and at == e.size)}
