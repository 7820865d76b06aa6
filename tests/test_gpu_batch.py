"""Batched form: many inputs of uneven sizes and levels in one call; every
stream must be byte-identical to compressing that input alone (plain form and
oracle), with blocks of level * 100,000 bytes."""
import bz2

import numpy as np
import pytest

import oracle
import bzip2gpu_b200 as B
import bzip2gpu_b200.workloads as W

pytestmark = pytest.mark.gpu


def _inputs():
    items = [(x.data, x.level) for x in W.batch_inputs(count=24, seed=0xB2C2, max_size=3 << 20)]
    items += [(np.zeros(0, np.uint8), 9), (np.array([7], np.uint8), 1),
              (W.small_markov(300000, seed=5), 3),      # exact multiple of its block size
              (np.zeros(250000, np.uint8), 2)]
    return items


def test_batch_streams_equal_single_stream_compression(torch_cuda):
    items = _inputs()
    data = [a for a, _ in items]
    levels = [lv for _, lv in items]
    streams = B.compress_batch(data, levels)
    assert len(streams) == len(items)
    for (a, lv), s in zip(items, streams):
        s = bytes(s)
        ref = oracle.compress(a, lv, lv * 100000, threads=8)
        assert s == ref
        assert s == B.compress(a, lv, lv * 100000)
        fits = all(oracle.rle1(a[i:i + lv * 100000]).size <= lv * 100000
                   for i in range(0, a.size, lv * 100000))
        if fits:
            assert bz2.decompress(s) == a.tobytes()


def test_batch_from_device_memory(torch_cuda):
    items = _inputs()[:10]
    d = [torch_cuda.from_numpy(np.ascontiguousarray(a)).cuda() for a, _ in items]
    streams = B.compress_batch(d, [lv for _, lv in items], on_device=True)
    for (a, lv), s in zip(items, streams):
        assert bytes(s) == oracle.compress(a, lv, lv * 100000)


@pytest.mark.parametrize("table", [
    [{"max_block_len": 300000, "slab_blocks": 3, "workers": 2},
     {"max_block_len": 900000, "slab_blocks": 1, "workers": 5}],
    [{"max_block_len": 900000, "slab_blocks": 1024, "workers": 1}],
])
def test_batch_tuning_changes_no_byte(torch_cuda, table):
    # slab shapes from a tuning table (tiny slabs, single-block slabs, slabs as
    # large as the workspace allows, one worker) give the same streams
    items = _inputs()
    data = [a for a, _ in items]
    levels = [lv for _, lv in items]
    ref = [bytes(s) for s in B.compress_batch(data, levels)]
    try:
        B.set_batch_tuning(table)
        got = [bytes(s) for s in B.compress_batch(data, levels)]
    finally:
        B.set_batch_tuning([])
        B._tuning_applied = False
    assert got == ref


def test_committed_tuning_table_is_well_formed():
    import json
    if not B.TUNING_FILE.exists():
        pytest.skip("no tuning table committed")
    t = json.loads(B.TUNING_FILE.read_text())["table"]
    assert t and all(e["max_block_len"] > 0 and 1 <= e["slab_blocks"] <= 1024 and
                     e["workers"] >= 1 for e in t)
