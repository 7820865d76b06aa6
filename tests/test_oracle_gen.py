"""The oracle's workload generator (oracle/gen_oracle.c) against the product
library's host generator (bzip2gpu_b200/csrc/gen.cu): the same bytes for the
same arguments.  The CPU reference timing builds its sample with the oracle's
generator, so this pin is what makes both arms compress the same stream."""
import numpy as np
import pytest

import bzip2gpu_b200 as B
import bzip2gpu_b200.workloads as W
import oracle

CASES = [
    (0xB2C0, np.arange(0x20, 0x80, dtype=np.uint8), 0.3, 0.02, 4, 300, 300_001),
    (7, np.array([3, 200], np.uint8), 0.05, 0.01, 4, 255, 200_000),
    (0xB2C4 * 1000003 + 5, np.arange(256, dtype=np.uint8), 4.9, 0.02, 4, 300, 131_073),
    (11, np.array([65], np.uint8), 1.0, 0.5, 1, 1, 65_536 * 3 + 17),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_markov_bytes_equal_product_generator(case):
    seed, alph, alpha, p_run, lo, hi, n = CASES[case]
    want = B.gen_markov(n, seed, alph, alpha, p_run, lo, hi)
    got = oracle.gen_markov(n, seed, alph, alpha, p_run, lo, hi)
    assert np.array_equal(got, want)


def test_uniform_bytes_equal_product_generator():
    assert np.array_equal(oracle.gen_uniform(1_000_003, 0xB2C1C),
                          B.gen_uniform(1_000_003, 0xB2C1C))


def test_large_stream_across_a_segment_border():
    n = (64 << 20) + (1 << 20)
    got = oracle.large_stream(n)
    want = W.large_stream(n, device=False)
    assert np.array_equal(got, want)


def test_bad_arguments_rejected():
    with pytest.raises(ValueError):
        oracle.gen_markov(10, 1, np.zeros(0, np.uint8), 1.0, 0.0, 4, 10)
