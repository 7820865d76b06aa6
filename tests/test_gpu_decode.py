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
