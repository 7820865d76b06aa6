"""Checker tools of the oracle: the bounded sample of the large stream, and
libbz2 decoding of a long stream block by block (each block re-wrapped as a
stream of its own) -- the way the benchmark proves its multi-GB streams
round-trip."""
import bz2

import numpy as np

import oracle


def test_sample_is_the_streams_own_bytes():
    n = (64 << 20) * 2 + 5
    full = oracle.large_stream(n)
    s = oracle.large_stream_sample(n, per_segment=100_000)
    assert s.size == 200_005
    assert np.array_equal(s[:100_000], full[:100_000])
    assert np.array_equal(s[100_000:200_000], full[64 << 20:(64 << 20) + 100_000])
    assert np.array_equal(s[200_000:], full[128 << 20:])


def test_libbz2_block_decode_of_oracle_and_libbz2_streams():
    a = oracle.large_stream(6 << 20)
    r = oracle.libbz2_matches(oracle.compress(a, 9, threads=4), a)
    assert r == {"blocks": 7, "bytes": a.size, "identical": True}
    r = oracle.libbz2_matches(bz2.compress(a.tobytes(), 2), a)
    assert r["identical"] and r["blocks"] > 7


def test_libbz2_block_decode_detects_damage_and_length():
    a = oracle.large_stream(2 << 20)
    z = bytearray(bz2.compress(a.tobytes(), 1))
    assert not oracle.libbz2_matches(z, a[:-1])["identical"]
    z[len(z) // 2] ^= 0x10
    assert not oracle.libbz2_matches(bytes(z), a)["identical"]
