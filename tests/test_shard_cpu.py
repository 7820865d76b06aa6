"""One stream over several ranks: the exchange of bzip2gpu_b200/shard.py on
the CPU with gloo (world sizes 2 and 3), the parts and the assembly supplied
by the oracle.  Rank 0's stream must equal the oracle's stream of the whole
input."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import oracle
import bzip2gpu_b200.shard as SH
import bzip2gpu_b200.workloads as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _part_fn(data, block_bytes):
    p, bits, fold, nb = oracle.compress_part(np.asarray(data), block_bytes)
    pad = (-p.size) % 4
    return torch.from_numpy(np.concatenate([p, np.zeros(pad, np.uint8)])), bits, fold, nb


def _assemble_fn(parts, bits, folds, nblocks, level):
    return oracle.assemble([p.numpy() for p in parts], bits, folds, nblocks, level)


def _worker(rank, world, port, case, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        data, level, bb = case
        out = SH.compress_sharded(data, level, bb, part_fn=_part_fn, assemble_fn=_assemble_fn)
        if rank == 0:
            q.put(out)
    finally:
        dist.destroy_process_group()


CASES = {
    "markov_uneven": (W.small_markov(1000001, seed=51), 9, 90000),
    "two_blocks_three_ranks": (W.small_markov(150000, seed=52), 5, 100000),
    "one_block": (W.small_markov(5000, seed=53), 9, 900000),
    "empty": (np.zeros(0, np.uint8), 9, 900000),
}


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", sorted(CASES))
def test_sharded_stream_equals_single_stream(world, name):
    data, level, bb = CASES[name]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, (data, level, bb), q))
             for r in range(world)]
    for p in procs:
        p.start()
    out = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == oracle.compress(data, level, bb)


def test_block_ranges_cover_blocks_in_order():
    for n, bb, world in [(10, 3, 3), (0, 5, 2), (7, 3, 4), (900000 * 7 + 5, 900000, 3)]:
        r = SH.block_ranges(n, bb, world)
        assert len(r) == world and r[0][0] == 0 and r[-1][1] == n
        assert all(a <= b for a, b in r) and all(r[i][1] == r[i + 1][0] for i in range(world - 1))
        assert all(a % bb == 0 or a == n for a, _ in r)
        counts = [-(-(b - a) // bb) for a, b in r]
        assert max(counts) - min(counts) <= 1
