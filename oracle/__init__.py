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
            (HERE / f).stat().st_mtime for f in ("bz2_oracle.c", "bz2_oracle.h")):
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


def huffman_build(syms, n_in_use: int):
    """(len[6,258], code[6,258], selectors, n_groups)"""
    s = np.ascontiguousarray(syms, dtype=np.uint16)
    ln = np.zeros((G, A), np.uint8)
    code = np.zeros((G, A), np.int32)
    sel = np.zeros(s.size // 50 + 2, np.uint8)
    ng = _i()
    nsel = lib().orc_huffman_build(s.ctypes.data, s.size, n_in_use, ln.ctypes.data,
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

