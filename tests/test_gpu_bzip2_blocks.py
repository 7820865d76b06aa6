"""bzip2 1.0.8's block format (B.BZIP2_BLOCKS): the GPU split equals the
oracle's restatement of libbz2's split, and the streams are byte-identical to
libbz2's (Python's bz2 module) at every level; periodic blocks, where only the
origPtr among equal rotations may differ, round-trip."""
import bz2

import numpy as np
import pytest

import bzip2gpu_b200 as B
import bzip2gpu_b200.workloads as W
import oracle as O

pytestmark = pytest.mark.gpu


def _runs(seed: int, n_runs: int, lo: int, hi: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.repeat(rng.integers(0, 60, n_runs).astype(np.uint8),
                     rng.integers(lo, hi, n_runs))


def _text(lines: int) -> np.ndarray:
    return np.frombuffer(b"".join(b"record %d: value %d, flag %d\n" % (i, i * 7919 % 10007, i % 3)
                                  for i in range(lines)), np.uint8)


CASES = {
    "markov": lambda: W.small_markov(2_500_000, seed=101),
    "text": lambda: _text(60000),
    "long_runs": lambda: _runs(102, 30000, 1, 700),   # runs across block cuts
    "exact4": lambda: np.repeat(np.random.default_rng(103).integers(0, 256, 400000)
                                .astype(np.uint8), 4),
    "short_runs": lambda: _runs(104, 500000, 1, 6),
    "uniform": lambda: B.gen_uniform(1_200_000, 105),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("level", [1, 4, 9])
def test_split_matches_oracle(torch_cuda, name, level):
    a = CASES[name]()
    d = torch_cuda.from_numpy(a.copy()).cuda()
    assert np.array_equal(B.bzip2_split(d, level), O.bzip2_split(a, level))


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("level", [1, 9])
def test_streams_identical_to_libbz2(torch_cuda, name, level):
    a = CASES[name]()
    s = B.compress(a, level, B.BZIP2_BLOCKS)
    assert s == bz2.compress(a.tobytes(), level)
    assert B.decompress(s) == a.tobytes()


def test_every_level_and_the_device_forms(torch_cuda):
    torch = torch_cuda
    a = np.concatenate([_text(20000), W.small_markov(600_000, seed=106), _runs(107, 4000, 1, 400)])
    d = torch.from_numpy(a.copy()).cuda()
    for level in range(1, 10):
        want = bz2.compress(a.tobytes(), level)
        assert B.compress(a, level, B.BZIP2_BLOCKS) == want, level
        assert B.compress_device(d, level, B.BZIP2_BLOCKS) == want, level
    out = np.zeros(B.compress_bound(a.size, B.BZIP2_BLOCKS), np.uint8)
    n = B.compress_into(a, out, 9, B.BZIP2_BLOCKS)
    assert out[:n].tobytes() == bz2.compress(a.tobytes(), 9)


def test_tiny_and_empty_inputs(torch_cuda):
    for raw in [b"", b"a", b"ab", b"aaaa", b"aaaaa", b"hello world!\n", bytes(range(256))]:
        a = np.frombuffer(raw, np.uint8)
        assert B.compress(a, 9, B.BZIP2_BLOCKS) == bz2.compress(raw, 9), raw


def test_long_zero_runs_many_blocks(torch_cuda):
    # 64 MiB of zeros at level 1: blocks of about 5 MB of raw bytes, each a
    # periodic RLE1 block (libbz2 may pick another origPtr among its equal
    # rotations), so the stream is checked against the oracle and decoded
    torch = torch_cuda
    n = 64 << 20
    d = torch.zeros(n, dtype=torch.uint8, device="cuda")
    z = np.zeros(n, np.uint8)
    ends = B.bzip2_split(d, 1)
    assert np.array_equal(ends, O.bzip2_split(z, 1)) and len(ends) == 14
    s = B.compress_device(d, 1, B.BZIP2_BLOCKS)
    assert s == O.compress(z, 1, O.BZIP2_BLOCKS, threads=8)
    assert bz2.decompress(s) == bytes(n)


@pytest.mark.parametrize("name", ["ab", "period17"])
def test_periodic_blocks_round_trip(torch_cuda, name):
    a = np.tile(np.frombuffer(b"ab", np.uint8), 600000) if name == "ab" else W.periodic17(1_000_000)
    for level in (1, 9):
        s = B.compress(a, level, B.BZIP2_BLOCKS)
        assert bz2.decompress(s) == a.tobytes()
        assert B.decompress(s) == a.tobytes()
        # same bytes as the oracle (index order among equal rotations)
        assert s == O.compress(a, level, O.BZIP2_BLOCKS, threads=4)


def test_large_markov_stream(torch_cuda):
    d = W.large_stream(48 << 20, seed=0xB2C4 + 9, device=True)
    a = d.cpu().numpy()
    s = B.compress_device(d, 9, B.BZIP2_BLOCKS)
    assert s == bz2.compress(a.tobytes(), 9)


@pytest.mark.parametrize("seed", range(4))
def test_random_runs_equal_libbz2(torch_cuda, seed):
    # run lengths around the 4-byte threshold and the 255-byte cut, so block
    # cuts land inside and next to long runs (small blocks: levels 1-3)
    rng = np.random.default_rng(300 + seed)
    n_runs = int(rng.integers(20000, 60000))
    lens = rng.choice([1, 2, 3, 4, 5, 254, 255, 256, 259, 300, 510, 511, 1000],
                      size=n_runs, p=[.3, .15, .1, .1, .05, .04, .04, .04, .04, .04, .04, .03, .03])
    vals = rng.integers(0, int(rng.integers(2, 256)), n_runs).astype(np.uint8)
    a = np.repeat(vals, lens)
    level = int(rng.integers(1, 4))
    d = torch_cuda.from_numpy(a.copy()).cuda()
    assert np.array_equal(B.bzip2_split(d, level), O.bzip2_split(a, level))
    assert B.compress(a, level, B.BZIP2_BLOCKS) == bz2.compress(a.tobytes(), level)
