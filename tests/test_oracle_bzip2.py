"""The oracle's bzip2 1.0.8 mode (ORC_BZIP2_BLOCKS: libbz2's block split and
255-byte runs), pinned to libbz2 itself: its streams are byte-identical to
Python's bz2 module (libbz2 1.0.8) on inputs whose blocks have no equal
rotations, at every level, and its split has the properties of libbz2's."""
import bz2

import numpy as np
import pytest

import oracle as O
import bzip2gpu_b200.workloads as W


def _runs(seed, n_runs, lo, hi):
    rng = np.random.default_rng(seed)
    return np.repeat(rng.integers(0, 60, n_runs).astype(np.uint8), rng.integers(lo, hi, n_runs))


def _text(lines):
    return np.frombuffer(b"".join(b"record %d: value %d, flag %d\n" % (i, i * 7919 % 10007, i % 3)
                                  for i in range(lines)), np.uint8)


INPUTS = {
    "markov": lambda: W.small_markov(1_500_000, seed=201),
    "text": lambda: _text(50000),
    "long_runs": lambda: _runs(202, 20000, 1, 700),
    "exact4": lambda: np.repeat(np.random.default_rng(203).integers(0, 256, 300000)
                                .astype(np.uint8), 4),
    "tiny": lambda: np.frombuffer(b"hello world!\n", np.uint8),
    "empty": lambda: np.zeros(0, np.uint8),
}


@pytest.mark.parametrize("name", sorted(INPUTS))
@pytest.mark.parametrize("level", [1, 2, 9])
def test_oracle_bzip2_mode_equals_libbz2(name, level):
    a = INPUTS[name]()
    assert O.compress(a, level, O.BZIP2_BLOCKS, threads=4) == bz2.compress(a.tobytes(), level)


@pytest.mark.parametrize("level", [1, 9])
def test_split_properties(level):
    a = np.concatenate([_text(30000), _runs(204, 8000, 1, 900)])
    ends = O.bzip2_split(a, level)
    assert ends[-1] == a.size and np.all(np.diff(ends) > 0)
    max_written = 100000 * level - 19
    start = 0
    for e in ends:
        m = O.rle1_cut(a[start:e], 255).size
        # a block's RLE1 output stays within the level's 100000 * level bytes
        assert m <= max_written + 4
        if e != a.size:
            assert m >= max_written  # cut only once the limit is reached
        start = e


def test_run_cut_255_differs_from_259_only_on_long_runs():
    a = np.repeat(np.arange(10, dtype=np.uint8), 300)
    r255, r259 = O.rle1_cut(a, 255), O.rle1(a)
    assert r255.size == 10 * (5 + 5) and r259.size == 10 * (5 + 5)
    assert list(r255[:10]) == [0, 0, 0, 0, 251, 0, 0, 0, 0, 41]
    assert list(r259[:10]) == [0, 0, 0, 0, 255, 0, 0, 0, 0, 37]


@pytest.mark.parametrize("level", [1, 9])
def test_bzip2_format_bounds_hold(level):
    # the library's host-side bounds for BZ2G_BZIP2_BLOCKS (no GPU needed):
    # the stream bound covers the oracle's stream, and the split bound its
    # block count, on inputs that make many blocks or expand under RLE1
    import bzip2gpu_b200 as B
    rng = np.random.default_rng(205)
    cases = [np.repeat(rng.integers(0, 256, 250000).astype(np.uint8), 4),  # RLE1 expands 5/4
             rng.integers(0, 256, 600000).astype(np.uint8),
             np.zeros(3_000_000, np.uint8)]
    for a in cases:
        s = O.compress(a, level, O.BZIP2_BLOCKS, threads=4)
        assert len(s) <= B.compress_bound(a.size, B.BZIP2_BLOCKS)
        assert O.bzip2_split(a, level).size <= B.lib().bz2g_bzip2_split_bound(a.size, level)


@pytest.mark.parametrize("seed", range(8))
def test_oracle_bzip2_mode_random_runs_equal_libbz2(seed):
    # run lengths around the 4-byte threshold and the 255-byte cut, mixed
    # with literals, so block cuts land inside and next to long runs
    rng = np.random.default_rng(300 + seed)
    n_runs = int(rng.integers(20000, 60000))
    lens = rng.choice([1, 2, 3, 4, 5, 254, 255, 256, 259, 300, 510, 511, 1000],
                      size=n_runs, p=[.3, .15, .1, .1, .05, .04, .04, .04, .04, .04, .04, .03, .03])
    vals = rng.integers(0, int(rng.integers(2, 256)), n_runs).astype(np.uint8)
    a = np.repeat(vals, lens)
    level = int(rng.integers(1, 4))
    assert O.compress(a, level, O.BZIP2_BLOCKS, threads=4) == bz2.compress(a.tobytes(), level)
