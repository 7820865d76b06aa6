"""One stream over several GPUs, the GPU pieces: parts compressed by the
library and spliced by bz2g_assemble equal the single-GPU stream (and the
oracle's); a one-rank process group runs bzip2gpu_b200.shard end to end."""
import os
import socket

import numpy as np
import pytest

import oracle
import bzip2gpu_b200 as B
import bzip2gpu_b200.shard as SH
import bzip2gpu_b200.workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["markov_3parts", "zeros_2parts", "uneven_5parts", "empty_part"])
def test_parts_assemble_to_the_single_stream(torch_cuda, case):
    data, bb, k = {
        "markov_3parts": (W.small_markov(4000000, seed=61), 900000, 3),
        "zeros_2parts": (np.zeros(2000000, np.uint8), 300000, 2),
        "uneven_5parts": (W.small_markov(1234567, seed=62), 99999, 5),
        "empty_part": (W.small_markov(150000, seed=63), 100000, 3),
    }[case]
    parts, bits, folds, nbs = [], [], [], []
    for a, b in SH.block_ranges(data.size, bb, k):
        p, n, f, m = B.compress_part(data[a:b], bb)
        parts.append(p)
        bits.append(n)
        folds.append(f)
        nbs.append(m)
    s = B.assemble(parts, bits, folds, nbs, 9)
    assert s == B.compress(data, 9, bb) == oracle.compress(data, 9, bb, threads=8)


def test_part_from_device_input(torch_cuda):
    data = W.small_markov(2500000, seed=64)
    d = torch_cuda.from_numpy(data).cuda()
    p1, b1, f1, n1 = B.compress_part(d[:1800000], 900000)
    p2, b2, f2, n2 = B.compress_part(d[1800000:], 900000)
    assert B.assemble([p1, p2], [b1, b2], [f1, f2], [n1, n2], 9) == B.compress(data, 9)


def test_one_rank_group(torch_cuda):
    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        data = W.small_markov(2000000, seed=65)
        assert SH.compress_sharded(data, 9, 900000) == B.compress(data, 9)
    finally:
        dist.destroy_process_group()
