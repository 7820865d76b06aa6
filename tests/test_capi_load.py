"""The native library loads on a machine without a GPU and exports every
function declared in include/*.h (no compute calls here)."""
import re
import subprocess
from pathlib import Path

import bzip2gpu_b200 as B

ROOT = Path(__file__).resolve().parents[1]


def _exported():
    out = subprocess.run(["nm", "-D", "--defined-only", str(B.lib_path())], capture_output=True,
                         text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_library_loads():
    L = B.lib()
    assert L.bz2g_version() >= 1
    assert B.compress_bound(1000) > 1000


def test_c_abi_symbols_exported():
    decl = (ROOT / "include" / "bz2g.h").read_text()
    names = set(re.findall(r"\b(bz2g_[a-z0-9_]+)\s*\(", decl))
    assert len(names) >= 20
    missing = names - _exported()
    assert not missing, missing


def test_cpp_dropin_symbols_exported():
    # demangled names of the reference's include/compression.h, io.h, cli.h, crc32.h
    out = subprocess.run(["nm", "-DC", "--defined-only", str(B.lib_path())], capture_output=True,
                         text=True, check=True).stdout
    for sig in ["rle1_compress(unsigned char const*, int, unsigned char*&, CUstream_st*)",
                "rle2_compress(unsigned char const*, int, unsigned short*, unsigned int*, int, CUstream_st*)",
                "make_symbols_table(unsigned char const*, int, unsigned char*&, CUstream_st*)",
                "fmtf(unsigned char const*, int const*, int, unsigned char*&, int&, bool*, CUstream_st*)",
                "huffman_build_trees(unsigned short*, int, int, unsigned char (*) [258], int (*) [258], unsigned char*&, int&, CUstream_st*)",
                "fbwt(unsigned char const*, int, int*&, CUstream_st*)",
                "huffman_encode(unsigned short*, int, int, unsigned int*&, unsigned char (*) [258], int (*) [258], unsigned char*, int, int, CUstream_st*)",
                "count_frequencies(unsigned short*, int, int*)",
                "BZFileInputStream::fetch(unsigned char*&, int&)",
                "parse_args(int, char**)",
                "bzip2_crc32(unsigned char const*, unsigned long)"]:
        assert sig in out, sig
    assert "bzip2_gpu_compress(BZFileInputStream&, int, std::vector<unsigned char, std::allocator<unsigned char> >&)" in out


def test_cli_help_runs_without_gpu():
    cli = B.lib_path().parent / "bzip2gpu"
    r = subprocess.run([str(cli), "-h"], capture_output=True, text=True)
    assert r.returncode == 0 and "--best" in r.stdout


def test_engine_shape_host_logic():
    # bz2g_set_engine / bz2g_get_engine only touch host state (no CUDA call)
    shape = B.get_engine()
    assert shape == (384, 4)
    try:
        B.set_engine(16, 2)
        assert B.get_engine() == (16, 2)
        B.set_engine(0, 3)  # 0 keeps the current value
        assert B.get_engine() == (16, 3)
        B.set_engine(32, 0)
        assert B.get_engine() == (32, 3)
        try:
            B.set_engine(-1, 1)
        except Exception:
            pass
        else:
            raise AssertionError("a negative engine shape was accepted")
        assert B.get_engine() == (32, 3)
    finally:
        B.set_engine(*shape)
    assert B.get_engine() == shape


def test_batch_tuning_table_validation():
    # the committed table is well formed and accepted; bad entries are refused
    import json
    table = json.loads(B.TUNING_FILE.read_text())["table"]
    assert [t["max_block_len"] for t in table] == sorted(t["max_block_len"] for t in table)
    assert all(t["slab_blocks"] > 0 and t["workers"] > 0 for t in table)
    B.set_batch_tuning(table)
    try:
        B.set_batch_tuning([{"max_block_len": 900000, "slab_blocks": 0, "workers": 4}])
    except Exception:
        pass
    else:
        raise AssertionError("a zero slab size was accepted")
    B.set_batch_tuning(table)  # the committed table stays in force
