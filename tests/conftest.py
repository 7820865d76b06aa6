"""Shared test set-up: the `gpu` marker, repo root on sys.path, and the
reference tests' glibc rand() input generators."""
from __future__ import annotations

import ctypes
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


_libc = ctypes.CDLL("libc.so.6")


def glibc_rand(n: int) -> np.ndarray:
    """n successive glibc rand() values (after whatever srand was called)."""
    f = _libc.rand
    return np.fromiter((f() for _ in range(n)), dtype=np.int64, count=n)


def srand(seed: int) -> None:
    _libc.srand(seed)


def ref_rle1_input(max_run: int, n: int = 1000000) -> np.ndarray:
    """tests/compression/rle1.cu:34-47 of the reference (srand(2137))."""
    srand(2137)
    out = np.empty(n, np.uint8)
    chr_, reps, i = 0, 0, 0
    f = _libc.rand
    while i < n:
        if not reps:
            reps = f() % max_run + 1
            chr_ = (chr_ + f() % 100 + 1) & 255
        k = min(reps, n - i)
        out[i:i + k] = chr_
        i += k
        reps -= k
    return out


def ref_bwt_input(alphabet: int, n: int = 5000) -> np.ndarray:
    """tests/compression/fbwt.cu:26-31 of the reference."""
    srand(2137)
    return (glibc_rand(n) % alphabet).astype(np.uint8)


def ref_mtf_input(alphabet: int, n: int = 1000000) -> np.ndarray:
    """tests/compression/fmtf.cu:76-81 of the reference."""
    srand(2137)
    return (glibc_rand(n) % alphabet).astype(np.uint8)


def ref_rle2_input(max_run: int, n: int = 1000000) -> np.ndarray:
    """tests/compression/rle2.cu:35-46 of the reference."""
    srand(2137)
    out = np.empty(n, np.uint8)
    f = _libc.rand
    reps, i = 0, 0
    while i < n:
        if not reps:
            reps = f() % max_run + 1
            out[i] = f() % 256
        else:
            out[i] = out[i - 1]
        reps -= 1
        i += 1
    return out


def ref_rle2_incompressible(n: int = 1000000) -> np.ndarray:
    """tests/compression/rle2.cu:89-93 of the reference."""
    srand(2137)
    return (glibc_rand(n) % 255 + 1).astype(np.uint8)


def ref_huffman_input(n: int = 10000, alphabet: int = 15) -> np.ndarray:
    """tests/compression/huffman.cu:172-181 of the reference."""
    srand(2137)
    f = _libc.rand
    out = np.empty(n, np.uint16)
    shift = 0
    for i in range(n):
        if i % 50 == 0:
            shift = f() % 6
        out[i] = f() % (alphabet // 2) + shift
    return out


def table_size(a: np.ndarray) -> int:
    return int(np.unique(a).size)


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu-marked tests")
    return torch
