"""The reference's own unit tests run against this library, and the drop-in
C++ API driven the way the reference's main() drives it.

1. oracle/_ref/ref_unit_tests: the reference's tests/compression/*.cu and
   tests/io.cpp compiled unchanged against this project's include/ and linked
   to this library (its static archive, one CUDA runtime in the program as in
   the reference's own build; `make -C oracle ref-tests REF=<reference tree>`,
   with a small runner in place of GoogleTest).  They call rle1_compress,
   rle2_compress, fbwt, fmtf, make_symbols_table, huffman_build_trees,
   huffman_encode, count_frequencies (launched directly from the test) and
   BZFileInputStream, and check them against the reference tests' own CPU
   oracles.  The io test reads test_files/input_test_file, whose contents
   the test itself defines ("word0\\n" .. "word9\\n" in 6-byte chunks); it is
   written into a scratch directory here.
2. tests/cpp/dropin_harness.cpp: bzip2_gpu_compress over a BZFileInputStream,
   whose stream must equal bz2g_compress's, plus the crc32.h functions.
"""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import bzip2gpu_b200 as B
import oracle

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
RUNNER = ROOT / "oracle" / "_ref" / "ref_unit_tests"
LIBDIR = ROOT / "bzip2gpu_b200" / "_lib"


def test_reference_unit_tests_pass_on_this_library(tmp_path, torch_cuda):
    if not RUNNER.exists():
        pytest.skip("oracle/_ref/ref_unit_tests not built (make -C oracle ref-tests REF=...)")
    (tmp_path / "test_files").mkdir()
    (tmp_path / "test_files" / "input_test_file").write_text(
        "".join(f"word{i}\n" for i in range(10)))
    env = dict(os.environ, LD_LIBRARY_PATH=f"{LIBDIR}:{os.environ.get('LD_LIBRARY_PATH', '')}")
    r = subprocess.run([str(RUNNER)], cwd=tmp_path, env=env, capture_output=True, text=True,
                       timeout=600)
    print(r.stdout[-3000:])
    print(r.stderr[-3000:])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    ran = [ln.split()[-1] for ln in r.stdout.splitlines() if ln.startswith("[       OK ]")]
    # every active TEST of the reference's suite (the compress.cu ones are
    # commented out in the reference)
    want = {"compress.rle1_normal", "compress.rle1_incompressible", "compress.rle1_long_runs",
            "compress.rle2_normal", "compress.rle2_incompressible", "compress.rle2_long_runs",
            "compress.fbwt_normal", "compress.fbwt_small_alphabet",
            "compress.fbwt_single_character", "compress.mtf_symbol_table_generation",
            "compress.fmtf_normal", "compress.fmtf_small_alphabet",
            "compress.huffman_count_frequencies", "compress.huffman_tree_builder_stability",
            "compress.huffman_encoding", "io.file_input_stream"}
    assert want <= set(ran), sorted(want - set(ran))
    assert "0 failed" in r.stdout


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    out = tmp_path_factory.mktemp("harness") / "dropin_harness"
    cmd = ["nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           f"-I{ROOT / 'include'}", "-x", "cu", str(ROOT / "tests" / "cpp" / "dropin_harness.cpp"),
           "-o", str(out), f"-L{LIBDIR}", "-lbz2gpu_b200", "-Xlinker", f"-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


@pytest.mark.parametrize("case", ["markov_3_blocks", "tiny", "empty", "exact_block"])
def test_bzip2_gpu_compress_over_file_stream_equals_c_abi(tmp_path, harness, torch_cuda, case):
    data = {
        "markov_3_blocks": oracle.large_stream(2_500_000),
        "tiny": np.frombuffer(b"abracadabra\n", np.uint8),
        "empty": np.zeros(0, np.uint8),
        "exact_block": oracle.large_stream(900_000),
    }[case]
    src = tmp_path / "in.bin"
    dst = tmp_path / "out.bz2"
    data.tofile(src)
    r = subprocess.run([str(harness), str(src), "9", "900000", str(dst)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = dst.read_bytes()
    assert got == B.compress(data, 9)
    assert got == oracle.compress(data, 9, threads=4)
