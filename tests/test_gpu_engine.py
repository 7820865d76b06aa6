"""Engine shape and on-demand workspaces: a small call takes room for its own
blocks only, a larger call grows the workspaces, and every stream still
equals the oracle's; bz2g_get_engine reads back what bz2g_set_engine set."""
import numpy as np
import pytest

import oracle
import bzip2gpu_b200 as B
import bzip2gpu_b200.workloads as W

pytestmark = pytest.mark.gpu


def test_engine_shape_round_trips_and_workspaces_grow(torch_cuda):
    default = B.get_engine()
    assert default == (384, 4)
    try:
        B.set_engine(8, 2)
        assert B.get_engine() == (8, 2)
        B.set_engine(0, 3)  # 0 keeps the slab size
        assert B.get_engine() == (8, 3)
        # one block, then two slabs of blocks (the workspaces grow between
        # the calls), then one block again on the grown workspaces
        for n, seed in ((300000, 41), (12 * 900000 + 5, 42), (1000, 43)):
            data = W.small_markov(n, seed=seed)
            got = B.compress(data, 9, 900000)
            assert got == oracle.compress(data, 9, 900000)
    finally:
        B.set_engine(*default)
    assert B.get_engine() == default


def test_engine_rejects_negative_shape(torch_cuda):
    with pytest.raises(Exception):
        B.set_engine(-1, 2)
    assert B.get_engine() == (384, 4)
