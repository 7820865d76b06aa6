"""The GPU decompressor: round trips of this library's streams (the
reference's format included, whose blocks can exceed the header digit's size
and which libbz2 rejects), libbz2's own streams at every level (255-byte
runs, bzip2's block split), concatenated streams, and malformed streams
(errors, never a fault)."""
import bz2

import numpy as np
import pytest

import bzip2gpu_b200 as B
import bzip2gpu_b200.workloads as W

pytestmark = pytest.mark.gpu

CASES = {
    "empty": (np.zeros(0, np.uint8), 9, 900000),
    "one": (np.array([65], np.uint8), 9, 900000),
    "hello": (np.frombuffer(b"hello world!\n", np.uint8), 1, 900000),
    "markov_3blocks": (W.small_markov(2500000, seed=81), 9, 900000),
    "zeros": (np.zeros(2700000, np.uint8), 9, 900000),
    "uniform": (B.gen_uniform(1000000, 82), 5, 900000),  # m > 900,000 blocks
    "periodic17": (W.periodic17(1000000), 9, 900000),
    "small_blocks": (W.small_markov(200000, seed=83), 3, 1000),
    "odd_blocks": (W.small_markov(500000, seed=84), 9, 99999),
    "runs_255": (np.repeat(np.arange(200, dtype=np.uint8), 1000), 9, 900000),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_round_trip_own_streams(torch_cuda, name):
    a, level, bb = CASES[name]
    s = B.compress(a, level, bb)
    assert B.decompress(s) == a.tobytes()


@pytest.mark.parametrize("level", [1, 5, 9])
@pytest.mark.parametrize("name", ["markov_3blocks", "zeros", "uniform", "runs_255", "hello",
                                  "periodic17"])
def test_libbz2_streams(torch_cuda, name, level):
    a = CASES[name][0]
    assert B.decompress(bz2.compress(a.tobytes(), level)) == a.tobytes()


def test_concatenated_streams_and_device_input(torch_cuda):
    a = W.small_markov(1500000, seed=85)
    b = np.zeros(300000, np.uint8)
    s = B.compress(a, 9) + bz2.compress(b.tobytes(), 3) + B.compress(a[:1000], 1)
    want = a.tobytes() + b.tobytes() + a[:1000].tobytes()
    assert B.decompress(s) == want
    d = torch_cuda.from_numpy(np.frombuffer(s, np.uint8).copy()).cuda()
    assert B.decompress_device(d) == want


def test_learned_streams_round_trip(torch_cuda):
    import bzip2gpu_b200.selector as S
    S.load_default()
    B.set_selector("learned")
    try:
        a = W.small_markov(3000000, seed=86)
        s = B.compress(a, 9)
    finally:
        B.set_selector("plain")
    assert B.decompress(s) == a.tobytes()


def test_large_stream_round_trip(torch_cuda):
    # many blocks in several decode batches
    d = W.large_stream(300 << 20, seed=0xB2C4 + 5, device=True)
    s = B.compress_device(d, 9)
    assert B.decompress(s) == d.cpu().numpy().tobytes()


@pytest.mark.parametrize("how", ["flip_payload", "flip_crc", "truncate", "garbage", "no_eos"])
def test_malformed_streams_are_errors(torch_cuda, how):
    a = W.small_markov(400000, seed=87)
    s = bytearray(B.compress(a, 9))
    if how == "flip_payload":
        s[len(s) // 2] ^= 0x10
    elif how == "flip_crc":
        s[12] ^= 0x01  # block CRC
    elif how == "truncate":
        s = s[: len(s) - 40]
    elif how == "garbage":
        s = bytearray(b"BZh9" + bytes(np.random.default_rng(1).integers(0, 256, 5000, np.uint8)))
    else:
        s = s[:-10]
    with pytest.raises(B.Bz2gError):
        B.decompress(bytes(s))


def test_decompress_into_buffers(torch_cuda):
    torch = torch_cuda
    a = W.small_markov(2000000, seed=88)
    s = B.compress(a, 9)
    want = a.tobytes()
    out = np.empty(len(want), np.uint8)
    assert B.decompress_into(s, out) == len(want) and out.tobytes() == want
    pin = torch.empty(len(want) + 100, dtype=torch.uint8, pin_memory=True)
    assert B.decompress_into(s, pin) == len(want) and pin[: len(want)].numpy().tobytes() == want
    d_in = torch.from_numpy(np.frombuffer(s, np.uint8).copy()).cuda()
    d_out = torch.empty(len(want), dtype=torch.uint8, device="cuda")
    assert B.decompress_into(d_in, d_out) == len(want)
    assert d_out.cpu().numpy().tobytes() == want
    with pytest.raises(B.Bz2gError):
        B.decompress_into(s, np.empty(len(want) - 1, np.uint8))
    assert B.decompress(B.compress(np.zeros(0, np.uint8))) == b""
    assert B.decompress_into(B.compress(np.zeros(0, np.uint8)), np.empty(0, np.uint8)) == 0


def _count_equals_byte_runs(n_runs: int, seed: int) -> np.ndarray:
    # runs of 4 + b copies of byte b: every RLE1 count byte equals the byte
    # of its run, the case where a segment's entry state stays ambiguous
    rng = np.random.default_rng(seed)
    vals = rng.integers(0, 40, n_runs).astype(np.uint8)
    return np.repeat(vals, vals.astype(np.int64) + 4)


@pytest.mark.parametrize("batch", ["1", "3", "64"])
def test_small_decode_batches(torch_cuda, monkeypatch, batch):
    monkeypatch.setenv("BZ2G_DECODE_BATCH", batch)
    a = np.concatenate([W.small_markov(150000, seed=89), _count_equals_byte_runs(3000, 90)])
    s = B.compress(a, 3, 7000)  # 33 blocks
    assert B.decompress(s) == a.tobytes()
    out = np.empty(a.size, np.uint8)
    assert B.decompress_into(s, out) == a.size and np.array_equal(out, a)


@pytest.mark.parametrize("seed", [91, 92])
def test_rle1_segments_with_ambiguous_states(torch_cuda, seed):
    a = _count_equals_byte_runs(60000, seed)
    assert B.decompress(B.compress(a, 9)) == a.tobytes()
    assert B.decompress(bz2.compress(a.tobytes(), 9)) == a.tobytes()
    # single runs of every length around the 4-byte threshold and 259 cut
    b = np.concatenate([np.full(L, L % 251, np.uint8) for L in range(1, 600)])
    assert B.decompress(B.compress(b, 9)) == b.tobytes()
    assert B.decompress(bz2.compress(b.tobytes(), 1)) == b.tobytes()


@pytest.mark.parametrize("seed", range(4))
def test_libbz2_run_heavy_streams(torch_cuda, seed):
    # run lengths around 4, 255 and 259 mixed with literals: long RUNA/RUNB
    # zero runs, MTF batches of repeats, RLE1 count bytes near 255
    rng = np.random.default_rng(400 + seed)
    n_runs = int(rng.integers(20000, 60000))
    lens = rng.choice([1, 2, 3, 4, 5, 254, 255, 256, 259, 300, 510, 1000],
                      size=n_runs, p=[.3, .15, .1, .1, .05, .05, .05, .04, .04, .04, .04, .04])
    vals = rng.integers(0, int(rng.integers(2, 256)), n_runs).astype(np.uint8)
    a = np.repeat(vals, lens)
    for level in (1, 9):
        assert B.decompress(bz2.compress(a.tobytes(), level)) == a.tobytes()
        assert B.decompress(B.compress(a, level)) == a.tobytes()
