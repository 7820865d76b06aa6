"""bzip2gpu-b200: the bzip2gpu compression path on NVIDIA B200 (sm_100a).

Python view of the C-ABI in include/bz2g.h (libbz2gpu_b200.so, built in-tree by
``python -m bzip2gpu_b200.build``).  Whole-stream calls take host bytes;
per-stage calls take torch CUDA tensors as device memory and mirror the
reference's operators (include/compression.h of SebastianBoteroLeonik/bzip2gpu):
rle1_compress, fbwt, fmtf, make_symbols_table, rle2_compress,
huffman_build_trees, huffman_encode, count_frequencies, bzip2_crc32.

There is no CPU fallback: every call runs the CUDA library, and loading fails
loudly when it has not been built.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

__all__ = [
    "Bz2gError", "lib", "lib_path", "compress", "compress_device", "compress_bound",
    "set_engine", "get_engine", "compress_into", "compress_device_into", "compress_batch", "rle1", "crc32", "bwt", "mtf", "symbols_table", "rle2", "huffman_build",
    "huffman_encode", "count_frequencies", "gen_markov", "gen_uniform", "MAX_GROUPS",
    "MAX_ALPHA", "SELECTOR_PARAMS", "selector_load", "set_selector", "get_selector",
    "selector_logits", "huffman_build_learned", "selector_dataset", "compress_part",
    "assemble", "compress_file", "decompress", "decompress_device", "decompress_into",
    "bzip2_split", "BZIP2_BLOCKS",
]

# block_bytes value selecting bzip2 1.0.8's block format (blocks cut by RLE1
# length, runs cut at 255): streams byte-identical to libbz2's
BZIP2_BLOCKS = -1
MAX_GROUPS = 6
MAX_ALPHA = 258
SELECTOR_PARAMS = 139792
_LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libbz2gpu_b200.so"
_lib = None

_c = ctypes
_vp, _i, _u8p, _sz = _c.c_void_p, _c.c_int, _c.POINTER(_c.c_uint8), _c.c_size_t

_SIGS = {
    "bz2g_last_error": (_c.c_char_p, []),
    "bz2g_version": (_i, []),
    "bz2g_compress": (_i, [_vp, _sz, _i, _i, _c.POINTER(_u8p), _c.POINTER(_sz)]),
    "bz2g_compress_device": (_i, [_vp, _sz, _i, _i, _c.POINTER(_u8p), _c.POINTER(_sz)]),
    "bz2g_compress_into": (_i, [_vp, _sz, _i, _i, _vp, _sz, _c.POINTER(_sz)]),
    "bz2g_compress_device_into": (_i, [_vp, _sz, _i, _i, _vp, _sz, _c.POINTER(_sz)]),
    "bz2g_compress_bound": (_sz, [_sz, _i]),
    "bz2g_compress_batch": (_i, [_i, _vp, _vp, _vp, _vp, _i, _vp, _sz, _vp]),
    "bz2g_compress_batch_bound": (_sz, [_i, _vp, _vp, _vp]),
    "bz2g_free": (None, [_vp]),
    "bz2g_set_engine": (_i, [_i, _i]),
    "bz2g_get_engine": (_i, [_c.POINTER(_i), _c.POINTER(_i)]),
    "bz2g_set_batch_tuning": (_i, [_i, _vp, _vp, _vp]),
    "bz2g_set_timing": (_i, [_i]),
    "bz2g_last_stats": (_i, [_c.POINTER(_c.c_double), _i]),
    "bz2g_launch_count": (_c.c_int64, []),
    "bz2g_last_round_stats": (_i, [_c.POINTER(_c.c_double), _i]),
    "bz2g_rle1_bound": (_sz, [_sz]),
    "bz2g_rle1": (_i, [_vp, _i, _vp, _c.POINTER(_i), _vp]),
    "bz2g_crc32": (_i, [_vp, _sz, _c.POINTER(_c.c_uint32), _vp]),
    "bz2g_bwt": (_i, [_vp, _i, _vp, _vp]),
    "bz2g_mtf": (_i, [_vp, _vp, _i, _vp, _c.POINTER(_i), _vp, _c.POINTER(_i), _vp]),
    "bz2g_symbols_table": (_i, [_vp, _i, _vp, _c.POINTER(_i), _vp]),
    "bz2g_rle2": (_i, [_vp, _i, _i, _vp, _vp, _vp]),
    "bz2g_huffman_build": (_i, [_vp, _i, _i, _vp, _vp, _vp, _c.POINTER(_i), _c.POINTER(_i), _vp]),
    "bz2g_huffman_encode": (_i, [_vp, _i, _vp, _vp, _vp, _i, _i, _vp, _c.POINTER(_c.c_int64), _vp]),
    "bz2g_count_frequencies": (_i, [_vp, _i, _vp, _vp]),
    "bz2g_gen_markov": (_i, [_c.c_uint64, _vp, _i, _c.c_double, _c.c_double, _i, _i, _vp,
                             _c.c_int64, _i, _vp]),
    "bz2g_gen_uniform": (_i, [_c.c_uint64, _vp, _c.c_int64, _i, _vp]),
    "bz2g_compress_file": (_i, [_c.c_char_p, _c.c_char_p, _i, _i]),
    "bz2g_decompress": (_i, [_vp, _sz, _c.POINTER(_u8p), _c.POINTER(_sz)]),
    "bz2g_decompress_device": (_i, [_vp, _sz, _c.POINTER(_u8p), _c.POINTER(_sz)]),
    "bz2g_decompress_into": (_i, [_vp, _sz, _vp, _sz, _c.POINTER(_sz)]),
    "bz2g_bzip2_split": (_i, [_vp, _sz, _i, _vp, _sz, _c.POINTER(_sz), _vp]),
    "bz2g_bzip2_split_bound": (_sz, [_sz, _i]),
    "bz2g_decompress_device_into": (_i, [_vp, _sz, _vp, _sz, _c.POINTER(_sz)]),
    "bz2g_part_bound": (_sz, [_sz, _i]),
    "bz2g_compress_part": (_i, [_vp, _sz, _i, _i, _vp, _sz, _c.POINTER(_c.c_int64),
                                _c.POINTER(_c.c_uint32), _c.POINTER(_i)]),
    "bz2g_assemble": (_i, [_i, _vp, _vp, _vp, _vp, _i, _vp, _sz, _c.POINTER(_sz)]),
    "bz2g_selector_load": (_i, [_vp, _sz]),
    "bz2g_set_selector": (_i, [_i]),
    "bz2g_get_selector": (_i, []),
    "bz2g_selector_logits": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "bz2g_selector_wait_check": (_i, [_vp, _i, _vp, _c.c_uint64, _i, _vp]),
    "bz2g_huffman_build_learned": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _c.POINTER(_i),
                                        _c.POINTER(_i), _vp]),
    "bz2g_selector_dataset": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _c.c_int64,
                                   _c.POINTER(_c.c_int64)]),
    "bz2g_mlp_features": (_i, [_vp, _c.c_int64, _vp, _vp, _vp]),
    "bz2g_mlp_work_bytes": (_sz, [_i]),
    "bz2g_mlp_grads": (_i, [_vp, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bz2g_mlp_forward": (_i, [_vp, _vp, _i, _vp, _vp, _vp, _vp, _vp]),
    "bz2g_mlp_adam": (_i, [_vp, _vp, _vp, _vp, _vp, _c.c_float, _c.c_float, _c.c_float,
                           _c.c_float, _i, _vp]),
    "bz2g_mlp_to_bf16": (_i, [_vp, _vp, _vp]),
    "bz2g_mlp_status": (_i, [_vp]),
}


class Bz2gError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"bz2g error {code}: {msg}")
        self.code = code


def lib_path() -> Path:
    return _LIB_PATH


def lib():
    """The loaded native library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise RuntimeError(f"native library missing: {_LIB_PATH} "
                               "(build it with `python -m bzip2gpu_b200.build`)")
        L = ctypes.CDLL(str(_LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise Bz2gError(rc, lib().bz2g_last_error().decode(errors="replace"))


def _stream(stream) -> int | None:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return int(stream)


def _ptr(t) -> int:
    return t.data_ptr()


def _take(ptr, n: int) -> bytes:
    """Bytes of a library-allocated buffer (any size), then free it."""
    try:
        if n == 0:
            return b""
        addr = ctypes.cast(ptr, ctypes.c_void_p).value
        return np.ctypeslib.as_array((ctypes.c_uint8 * n).from_address(addr)).tobytes()
    finally:
        lib().bz2g_free(ptr)


# ------------------------------------------------------------ whole stream
def _host_view(data) -> tuple[np.ndarray, int]:
    a = np.frombuffer(data, dtype=np.uint8) if isinstance(data, (bytes, bytearray, memoryview)) \
        else np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)
    return a, a.ctypes.data


def compress(data, level: int = 9, block_bytes: int = 900000) -> bytes:
    """Whole .bz2 stream of host bytes (bytes / numpy uint8 / pinned tensor)."""
    if hasattr(data, "data_ptr") and not getattr(data, "is_cuda", False):
        ptr, n, keep = data.data_ptr(), data.numel(), data
    else:
        keep, ptr = _host_view(data)
        n = keep.size
    out = _u8p()
    ln = _sz()
    _check(lib().bz2g_compress(ptr if n else None, n, level, block_bytes, ctypes.byref(out),
                               ctypes.byref(ln)))
    return _take(out, ln.value)


def compress_into(data, out, level: int = 9, block_bytes: int = 900000) -> int:
    """Whole .bz2 stream of host bytes written into `out` (a host buffer: numpy
    array or CPU tensor; page-locked memory receives the device copies
    directly).  Returns the stream length; raises if `out` is too small."""
    if hasattr(data, "data_ptr") and not getattr(data, "is_cuda", False):
        ptr, n = data.data_ptr(), data.numel()
    else:
        keep, ptr = _host_view(data)
        n = keep.size
    if hasattr(out, "data_ptr"):
        optr, cap = out.data_ptr(), out.numel() * out.element_size()
    else:
        optr, cap = out.ctypes.data, out.nbytes
    ln = _sz()
    _check(lib().bz2g_compress_into(ptr if n else None, n, level, block_bytes, optr, cap,
                                    ctypes.byref(ln)))
    return ln.value


def compress_device_into(d_in, out, level: int = 9, block_bytes: int = 900000) -> int:
    """Whole .bz2 stream of a CUDA uint8 tensor written into host buffer `out`."""
    if hasattr(out, "data_ptr"):
        optr, cap = out.data_ptr(), out.numel() * out.element_size()
    else:
        optr, cap = out.ctypes.data, out.nbytes
    ln = _sz()
    n = d_in.numel()
    _check(lib().bz2g_compress_device_into(_ptr(d_in) if n else None, n, level, block_bytes,
                                           optr, cap, ctypes.byref(ln)))
    return ln.value


def compress_device(d_in, level: int = 9, block_bytes: int = 900000) -> bytes:
    """Whole .bz2 stream of a CUDA uint8 tensor."""
    out = _u8p()
    ln = _sz()
    n = d_in.numel()
    _check(lib().bz2g_compress_device(_ptr(d_in) if n else None, n, level, block_bytes,
                                      ctypes.byref(out), ctypes.byref(ln)))
    return _take(out, ln.value)


TUNING_FILE = Path(__file__).resolve().parent / "batch_tuning.json"
_tuning_applied = False


def set_batch_tuning(table) -> None:
    """Batched-form slab shapes by block length: entries {"max_block_len",
    "slab_blocks", "workers"} (bz2g_set_batch_tuning); an empty list restores
    the engine's own shape."""
    global _tuning_applied
    n = len(table)
    arr = [(ctypes.c_int * max(n, 1))(*[int(e[k]) for e in table])
           for k in ("max_block_len", "slab_blocks", "workers")]
    _check(lib().bz2g_set_batch_tuning(n, *arr))
    _tuning_applied = True


def _apply_committed_tuning() -> None:
    """The measured table (bzip2gpu_b200/batch_tuning.json, written by
    bzip2gpu_b200.autotune), applied once before the first batched call."""
    if _tuning_applied:
        return
    if TUNING_FILE.exists():
        import json
        set_batch_tuning(json.loads(TUNING_FILE.read_text())["table"])
    else:
        set_batch_tuning([])


def compress_batch(inputs, levels, block_bytes=None, out=None, on_device=False):
    """Batched form: a list of inputs (host arrays/bytes, or CUDA tensors with
    on_device=True) -> list of .bz2 streams (memoryviews into one buffer).
    Block size per input: block_bytes[i], or levels[i] * 100000.  Slab shapes
    follow the committed tuning table unless set_batch_tuning() chose one."""
    _apply_committed_tuning()
    count = len(inputs)
    keep = []
    ptrs = (ctypes.c_void_p * max(count, 1))()
    sizes = (ctypes.c_size_t * max(count, 1))()
    lv = (ctypes.c_int * max(count, 1))(*[int(x) for x in levels])
    bb = None
    if block_bytes is not None:
        bb = (ctypes.c_int * max(count, 1))(*[int(x) for x in block_bytes])
    for i, x in enumerate(inputs):
        if on_device:
            ptrs[i], sizes[i] = x.data_ptr(), x.numel()
        else:
            a, p = _host_view(x)
            keep.append(a)
            ptrs[i], sizes[i] = p, a.size
    cap = lib().bz2g_compress_batch_bound(count, sizes, lv, bb)
    if out is None:
        out = np.empty(cap, np.uint8)
    optr = out.data_ptr() if hasattr(out, "data_ptr") else out.ctypes.data
    ocap = out.numel() if hasattr(out, "numel") else out.nbytes
    offs = (ctypes.c_size_t * (count + 1))()
    _check(lib().bz2g_compress_batch(count, ptrs, sizes, lv, bb, int(on_device), optr, ocap,
                                     offs))
    buf = memoryview(out.numpy() if hasattr(out, "numpy") else out)
    return [buf[offs[i]:offs[i + 1]] for i in range(count)]


def decompress(data) -> bytes:
    """Decode a .bz2 stream (host bytes) on the GPU."""
    keep, ptr = _host_view(data)
    out = _u8p()
    ln = _sz()
    _check(lib().bz2g_decompress(ptr if keep.size else None, keep.size, ctypes.byref(out),
                                 ctypes.byref(ln)))
    return _take(out, ln.value)


def decompress_device(d_in) -> bytes:
    """Decode a .bz2 stream held in a CUDA uint8 tensor."""
    out = _u8p()
    ln = _sz()
    _check(lib().bz2g_decompress_device(_ptr(d_in), d_in.numel(), ctypes.byref(out),
                                        ctypes.byref(ln)))
    return _take(out, ln.value)


def bzip2_split(d_in, level: int = 9) -> np.ndarray:
    """Block end offsets of bzip2 1.0.8's split of a CUDA uint8 tensor."""
    n = d_in.numel()
    cap = lib().bz2g_bzip2_split_bound(n, level)
    ends = np.zeros(max(cap, 1), np.int64)
    cnt = _sz()
    _check(lib().bz2g_bzip2_split(_ptr(d_in) if n else None, n, level, ends.ctypes.data, cap,
                                  ctypes.byref(cnt), _stream(None)))
    return ends[: cnt.value].copy()


def decompress_into(data, out) -> int:
    """Decode a .bz2 stream into a preallocated buffer; returns the decoded
    length (raises if `out` is too small).  `data` and `out` are host buffers
    (bytes, numpy arrays, CPU tensors; page-locked memory is copied directly)
    or CUDA uint8 tensors, in any combination."""
    ln = _sz()
    if hasattr(data, "data_ptr"):
        src, n = data.data_ptr(), data.numel()
        fn = lib().bz2g_decompress_device_into if data.is_cuda else lib().bz2g_decompress_into
    else:
        keep, src = _host_view(data)
        n, fn = keep.size, lib().bz2g_decompress_into
    if hasattr(out, "data_ptr"):
        dst, cap = out.data_ptr(), out.numel() * out.element_size()
    else:
        arr = out if isinstance(out, np.ndarray) else np.frombuffer(out, dtype=np.uint8)
        assert arr.flags.c_contiguous and arr.flags.writeable
        dst, cap = arr.ctypes.data, arr.nbytes
    _check(fn(src if n else None, n, dst if cap else None, cap, ctypes.byref(ln)))
    return ln.value


def compress_file(in_path, out_path, level: int = 9, group_blocks: int = 0) -> None:
    """Stream a file (None: stdin) into a .bz2 file (None: stdout) with bounded
    host memory: pinned input ring, groups of blocks on the GPU, output
    written as each group finishes (900,000-byte blocks, as the CLI)."""
    enc = lambda p: None if p is None else str(p).encode()
    _check(lib().bz2g_compress_file(enc(in_path), enc(out_path), level, group_blocks))


def compress_bound(n: int, block_bytes: int = 900000) -> int:
    return lib().bz2g_compress_bound(n, block_bytes)


def set_engine(slab_blocks: int = 0, workers: int = 0) -> None:
    _check(lib().bz2g_set_engine(slab_blocks, workers))


def get_engine() -> tuple[int, int]:
    """The engine shape of the whole-stream calls: (slab_blocks, workers)."""
    sb, nw = _c.c_int(0), _c.c_int(0)
    _check(lib().bz2g_get_engine(_c.byref(sb), _c.byref(nw)))
    return sb.value, nw.value


def set_timing(on: bool) -> None:
    _check(lib().bz2g_set_timing(int(on)))


STAT_FIELDS = ("blocks", "n", "m", "A", "s", "g", "bits", "ms_rle1", "ms_bwt", "ms_mtf",
               "ms_rle2", "ms_huffman", "ms_sizes", "ms_place", "scatter_launches",
               "scatter_ms", "scatter_bytes", "learned_blocks",
               "six_table_blocks")


def last_stats() -> dict:
    """Statistics of the last whole-stream call on this thread."""
    buf = (ctypes.c_double * len(STAT_FIELDS))()
    lib().bz2g_last_stats(buf, len(STAT_FIELDS))
    return dict(zip(STAT_FIELDS, list(buf)))


def last_round_stats() -> list[dict]:
    """BWT rounds of the last whole-stream call with timing on: per round its
    index (0: the first sort by 4-byte prefixes, standing for the doubling
    rounds with shift 1 and 2), the rotations the byte model charges to it
    (28 bytes each) and its device milliseconds summed over slabs."""
    buf = (ctypes.c_double * 96)()
    n = lib().bz2g_last_round_stats(buf, 96)
    return [{"round": int(buf[3 * r]), "active": int(buf[3 * r + 1]), "ms": buf[3 * r + 2]}
            for r in range(n)]


def launch_count() -> int:
    return int(lib().bz2g_launch_count())


def model_bytes(st: dict) -> float:
    """Algorithmic HBM bytes of the stage-boundary model:
    n + 10m + 28A + 14s + 5g + bits/8 (each stage reads its input once and
    writes its output once; a doubling round costs 28 bytes per rotation still
    in a non-singleton group)."""
    return st["n"] + 10 * st["m"] + 28 * st["A"] + 14 * st["s"] + 5 * st["g"] + st["bits"] / 8


# --------------------------------------------------------------- per stage
def rle1(d_in, stream=None):
    """rle1_compress: RLE1 (runs cut at 259) of a CUDA uint8 tensor."""
    import torch
    n = d_in.numel()
    out = torch.empty(lib().bz2g_rle1_bound(n), dtype=torch.uint8, device=d_in.device)
    m = _i()
    _check(lib().bz2g_rle1(_ptr(d_in), n, _ptr(out), ctypes.byref(m), _stream(stream)))
    return out[: m.value]


def crc32(d_in, stream=None) -> int:
    """bzip2_crc32 of a CUDA uint8 tensor."""
    c = ctypes.c_uint32()
    _check(lib().bz2g_crc32(_ptr(d_in), d_in.numel(), ctypes.byref(c), _stream(stream)))
    return c.value


def bwt(d_in, stream=None):
    """fbwt: int32 suffix array of the cyclic rotations."""
    import torch
    m = d_in.numel()
    sa = torch.empty(max(m, 1), dtype=torch.int32, device=d_in.device)
    _check(lib().bz2g_bwt(_ptr(d_in), m, _ptr(sa), _stream(stream)))
    return sa[:m]


def mtf(d_orig, d_sa, stream=None):
    """fmtf: (mtf values, origPtr, present[256] as uint8, nInUse)."""
    import torch
    m = d_orig.numel()
    out = torch.empty(max(m, 1), dtype=torch.uint8, device=d_orig.device)
    op = _i(-1)
    nu = _i()
    pres = np.zeros(256, np.uint8)
    _check(lib().bz2g_mtf(_ptr(d_orig), _ptr(d_sa), m, _ptr(out), ctypes.byref(op),
                          pres.ctypes.data, ctypes.byref(nu), _stream(stream)))
    return out[:m], op.value, pres, nu.value


def symbols_table(d_in, stream=None) -> np.ndarray:
    """make_symbols_table: ascending present byte values."""
    tbl = np.zeros(256, np.uint8)
    cnt = _i()
    _check(lib().bz2g_symbols_table(_ptr(d_in), d_in.numel(), tbl.ctypes.data, ctypes.byref(cnt),
                                    _stream(stream)))
    return tbl[: cnt.value].copy()


def rle2(d_mtf, table_size: int, stream=None):
    """rle2_compress: RUNA/RUNB symbols (int16 tensor holding uint16 values)."""
    import torch
    m = d_mtf.numel()
    out = torch.zeros(m + 1, dtype=torch.int16, device=d_mtf.device)
    ln = torch.zeros(1, dtype=torch.int32, device=d_mtf.device)
    _check(lib().bz2g_rle2(_ptr(d_mtf), m, table_size, _ptr(out), _ptr(ln), _stream(stream)))
    return out[: int(ln.item())]


def huffman_build(d_syms, n_in_use: int, stream=None):
    """huffman_build_trees: (len[6,258], code[6,258], selectors, n_groups)."""
    s = d_syms.numel()
    ln = np.full((MAX_GROUPS, MAX_ALPHA), 0, np.uint8)
    code = np.zeros((MAX_GROUPS, MAX_ALPHA), np.int32)
    sel = np.zeros(max((s + 49) // 50, 1), np.uint8)
    ns = _i()
    ng = _i()
    _check(lib().bz2g_huffman_build(_ptr(d_syms), s, n_in_use, ln.ctypes.data, code.ctypes.data,
                                    sel.ctypes.data, ctypes.byref(ns), ctypes.byref(ng),
                                    _stream(stream)))
    return ln, code, sel[: ns.value], ng.value


def huffman_encode(d_syms, len_tab: np.ndarray, code_tab: np.ndarray, d_sel, n_groups: int,
                   stream=None):
    """huffman_encode: (words as uint32 numpy array, total bits)."""
    import torch
    s = d_syms.numel()
    lt = np.ascontiguousarray(len_tab, dtype=np.uint8)
    ct = np.ascontiguousarray(code_tab, dtype=np.int32)
    words = torch.zeros((17 * s + 31) // 32 + 1, dtype=torch.int32, device=d_syms.device)
    bits = ctypes.c_int64()
    _check(lib().bz2g_huffman_encode(_ptr(d_syms), s, lt.ctypes.data, ct.ctypes.data, _ptr(d_sel),
                                     d_sel.numel(), n_groups, _ptr(words), ctypes.byref(bits),
                                     _stream(stream)))
    nw = (bits.value + 31) // 32
    return words[:nw].cpu().numpy().view(np.uint32), bits.value


def count_frequencies(d_syms, stream=None) -> np.ndarray:
    import torch
    f = torch.zeros(MAX_ALPHA, dtype=torch.int32, device=d_syms.device)
    _check(lib().bz2g_count_frequencies(_ptr(d_syms), d_syms.numel(), _ptr(f), _stream(stream)))
    return f.cpu().numpy()


# ------------------------------------------------------- synthetic inputs
def gen_markov(n: int, seed: int, alphabet, alpha: float, p_run: float, run_min: int,
               run_max: int, out=None, device: bool = False, stream=None):
    """Order-1 Markov bytes (bzip2gpu_b200/csrc/gen.cu).  Host numpy array, or
    a CUDA uint8 tensor when device=True (or `out` is one)."""
    alph = np.ascontiguousarray(alphabet, dtype=np.uint8)
    if out is None:
        if device:
            import torch
            out = torch.empty(n, dtype=torch.uint8, device="cuda")
        else:
            out = np.empty(n, np.uint8)
    on_dev = hasattr(out, "is_cuda") and out.is_cuda
    ptr = out.data_ptr() if hasattr(out, "data_ptr") else out.ctypes.data
    _check(lib().bz2g_gen_markov(seed & (2**64 - 1), alph.ctypes.data, alph.size, alpha, p_run,
                                 run_min, run_max, ptr, n, int(on_dev),
                                 _stream(stream) if on_dev else None))
    return out


def gen_uniform(n: int, seed: int, out=None, device: bool = False, stream=None):
    if out is None:
        if device:
            import torch
            out = torch.empty(n, dtype=torch.uint8, device="cuda")
        else:
            out = np.empty(n, np.uint8)
    on_dev = hasattr(out, "is_cuda") and out.is_cuda
    ptr = out.data_ptr() if hasattr(out, "data_ptr") else out.ctypes.data
    _check(lib().bz2g_gen_uniform(seed & (2**64 - 1), ptr, n, int(on_dev),
                                  _stream(stream) if on_dev else None))
    return out


# ------------------------------------------------- learned table selector
def selector_load(params) -> None:
    """Load selector parameters (flat fp32, SELECTOR_PARAMS values; layout in
    include/bz2g.h) on the current device."""
    p = np.ascontiguousarray(params, dtype=np.float32).reshape(-1)
    _check(lib().bz2g_selector_load(p.ctypes.data, p.size))


def set_selector(mode) -> None:
    """Table selector of the whole-stream calls: "plain" (0, the reference's),
    "learned" (1) or "one_pass" (2: the plain selector with a single
    selection pass, the learned form's measurement baseline)."""
    m = {"plain": 0, "learned": 1, "one_pass": 2}.get(mode, mode)
    _check(lib().bz2g_set_selector(int(m)))


def get_selector() -> str:
    return ("plain", "learned", "one_pass")[lib().bz2g_get_selector()]


def selector_logits(d_syms, d_params, stream=None):
    """The fused tensor-core selector over a symbol stream treated as one
    six-table block: (logits [groups, 6] float32 tensor, choices uint8 tensor)."""
    import torch
    s = d_syms.numel()
    g = (s + 49) // 50
    lg = torch.empty((g, 6), dtype=torch.float32, device=d_syms.device)
    sel = torch.empty(g, dtype=torch.uint8, device=d_syms.device)
    _check(lib().bz2g_selector_logits(_ptr(d_syms), s, _ptr(d_params), _ptr(lg), _ptr(sel),
                                      _stream(stream)))
    return lg, sel


ERR_TIMEOUT = 6


def selector_wait_check(d_syms, d_params, wait_limit_ns: int, withhold_weights: bool,
                        stream=None) -> None:
    """Failure-path check of the tensor-core selector kernel: every wait in
    it bounded by wait_limit_ns; withhold_weights makes the waits for the
    weights run out.  Raises Bz2gError (code ERR_TIMEOUT) when a wait ran out."""
    _check(lib().bz2g_selector_wait_check(_ptr(d_syms), d_syms.numel(), _ptr(d_params),
                                          int(wait_limit_ns), int(bool(withhold_weights)),
                                          _stream(stream)))


def huffman_build_learned(d_syms, n_in_use: int, d_params, stream=None):
    """huffman_build with the learned selector: (len, code, selectors, n_groups,
    the MLP's own choices)."""
    s = d_syms.numel()
    ln = np.zeros((MAX_GROUPS, MAX_ALPHA), np.uint8)
    code = np.zeros((MAX_GROUPS, MAX_ALPHA), np.int32)
    nsel = max((s + 49) // 50, 1)
    sel = np.zeros(nsel, np.uint8)
    msel = np.zeros(nsel, np.uint8)
    ns, ng = _i(), _i()
    _check(lib().bz2g_huffman_build_learned(_ptr(d_syms), s, n_in_use, _ptr(d_params),
                                            ln.ctypes.data, code.ctypes.data, sel.ctypes.data,
                                            msel.ctypes.data, ctypes.byref(ns), ctypes.byref(ng),
                                            _stream(stream)))
    return ln, code, sel[: ns.value], ng.value, msel[: ns.value]


def selector_dataset(d_inputs, levels, cap: int):
    """Training groups of the inputs (CUDA uint8 tensors): (group symbols
    [G, 50] uint16 tensor, plain-selector labels [G] uint8 tensor, groups
    available)."""
    import torch
    n = len(d_inputs)
    ptrs = (ctypes.c_void_p * max(n, 1))(*[t.data_ptr() for t in d_inputs])
    sizes = (ctypes.c_size_t * max(n, 1))(*[t.numel() for t in d_inputs])
    lv = (ctypes.c_int * max(n, 1))(*[int(x) for x in levels])
    syms = torch.empty((cap, 50), dtype=torch.int16, device="cuda")
    labels = torch.empty(cap, dtype=torch.uint8, device="cuda")
    got = ctypes.c_int64()
    _check(lib().bz2g_selector_dataset(n, ptrs, sizes, lv, _ptr(syms), _ptr(labels), cap,
                                       ctypes.byref(got)))
    k = min(cap, got.value)
    return syms[:k], labels[:k], got.value


# -------------------------------------------- one stream over several GPUs
def compress_part(data, block_bytes: int = 900000):
    """A part of a stream (whole blocks, no header, no end-of-stream marker)
    in device memory of the current device: (uint8 CUDA tensor whose length
    is a multiple of 4, bit count, CRC fold, blocks).  data: host bytes /
    numpy array, or a CUDA uint8 tensor."""
    import torch
    on_dev = hasattr(data, "is_cuda") and data.is_cuda
    if on_dev:
        ptr, n, keep = data.data_ptr(), data.numel(), data
    elif hasattr(data, "data_ptr"):
        ptr, n, keep = data.data_ptr(), data.numel(), data
    else:
        keep, ptr = _host_view(data)
        n = keep.size
    cap = lib().bz2g_part_bound(n, block_bytes)
    cap = (cap + 3) // 4 * 4
    part = torch.empty(cap, dtype=torch.uint8, device="cuda")
    bits, fold, nb = ctypes.c_int64(), ctypes.c_uint32(), _i()
    _check(lib().bz2g_compress_part(ptr if n else None, n, block_bytes, int(on_dev), _ptr(part),
                                    cap, ctypes.byref(bits), ctypes.byref(fold), ctypes.byref(nb)))
    used = ((bits.value + 7) // 8 + 3) // 4 * 4
    return part[:used], bits.value, fold.value, nb.value


def assemble(parts, bits, folds, nblocks, level: int = 9) -> bytes:
    """One .bz2 stream from parts (CUDA uint8 tensors on the current device,
    in stream order) with their bit counts, CRC folds and block counts."""
    k = len(parts)
    ptrs = (ctypes.c_void_p * max(k, 1))(*[p.data_ptr() for p in parts])
    b = (ctypes.c_int64 * max(k, 1))(*[int(x) for x in bits])
    f = (ctypes.c_uint32 * max(k, 1))(*[int(x) & 0xFFFFFFFF for x in folds])
    nb = (ctypes.c_int * max(k, 1))(*[int(x) for x in nblocks])
    cap = int(sum(int(x) for x in bits) // 8) + 64
    out = np.empty(cap, np.uint8)
    ln = _sz()
    _check(lib().bz2g_assemble(k, ptrs, b, f, nb, level, out.ctypes.data, cap, ctypes.byref(ln)))
    return out[: ln.value].tobytes()

