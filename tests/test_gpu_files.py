"""File streaming (bounded host memory): bz2g_compress_file and the CLI give
the same stream as one whole-buffer call, over several groups of blocks and
at the edges (empty file, exact block multiples, one byte); a missing input
is an error, not a hang."""
import subprocess

import numpy as np
import pytest

import oracle
import bzip2gpu_b200 as B
import bzip2gpu_b200.workloads as W

pytestmark = pytest.mark.gpu

CLI = B.lib_path().parent / "bzip2gpu"


@pytest.mark.parametrize("case,group", [("markov_7MB", 2), ("markov_7MB", 3), ("markov_7MB", 0),
                                        ("exact_2blocks", 1), ("one_byte", 1), ("empty", 1),
                                        ("zeros_5MB", 4)])
def test_compress_file_equals_whole_buffer(torch_cuda, tmp_path, case, group):
    data = {
        "markov_7MB": W.small_markov(7 * 1000 * 1000 + 13, seed=71),
        "exact_2blocks": W.small_markov(1800000, seed=72),
        "one_byte": np.array([0x41], np.uint8),
        "empty": np.zeros(0, np.uint8),
        "zeros_5MB": np.zeros(5 << 20, np.uint8),
    }[case]
    src = tmp_path / "in.bin"
    src.write_bytes(data.tobytes())
    dst = tmp_path / "out.bz2"
    B.compress_file(src, dst, 9, group)
    got = dst.read_bytes()
    assert got == B.compress(data, 9) == oracle.compress(data, 9, threads=8)


def test_missing_input_is_an_error(torch_cuda, tmp_path):
    with pytest.raises(B.Bz2gError):
        B.compress_file(tmp_path / "nope.bin", tmp_path / "o.bz2", 9)


def test_cli_file_stdout_and_stdin(torch_cuda, tmp_path):
    data = W.small_markov(2500000, seed=73)
    src = tmp_path / "f.dat"
    src.write_bytes(data.tobytes())
    r = subprocess.run([str(CLI), "-z", "-9", str(src)], capture_output=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "f.dat.bz2").read_bytes() == B.compress(data, 9)
    r = subprocess.run([str(CLI), "-c", "-5", str(src)], capture_output=True, timeout=300)
    assert r.returncode == 0 and r.stdout == B.compress(data, 5)
    r = subprocess.run([str(CLI)], input=data.tobytes(), capture_output=True, timeout=300)
    assert r.returncode == 0 and r.stdout == B.compress(data, 9)
    r = subprocess.run([str(CLI), str(tmp_path / "missing.dat")], capture_output=True, timeout=60)
    assert r.returncode != 0


def test_cli_bzip2_format_equals_libbz2(torch_cuda, tmp_path):
    # BZ2G_BZIP2_FORMAT=1: bzip2 1.0.8's block format, so every level gives
    # libbz2's own stream (levels 1..8 included)
    import bz2
    import os
    data = np.concatenate([W.small_markov(1500000, seed=74),
                           np.repeat(np.arange(40, dtype=np.uint8), 700)])
    src = tmp_path / "g.dat"
    src.write_bytes(data.tobytes())
    env = dict(os.environ, BZ2G_BZIP2_FORMAT="1")
    r = subprocess.run([str(CLI), "-z", "-1", str(src)], capture_output=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "g.dat.bz2").read_bytes() == bz2.compress(data.tobytes(), 1)
    r = subprocess.run([str(CLI), "-9"], input=data.tobytes(), capture_output=True, timeout=300,
                       env=env)
    assert r.returncode == 0 and r.stdout == bz2.compress(data.tobytes(), 9)
    r = subprocess.run([str(CLI), str(tmp_path / "missing.dat")], capture_output=True, timeout=60,
                       env=env)
    assert r.returncode != 0
