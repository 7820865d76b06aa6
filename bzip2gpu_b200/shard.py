"""One .bz2 stream compressed by several GPUs (one process per GPU,
torch.distributed).

The reference compresses every block independently (one host thread and
stream per block, src/compression/compress.cu:225-282) and only the stream
CRC fold and the bit-level concatenation tie the blocks together.  So rank r
compresses a contiguous range of whole blocks into a part
(bzip2gpu_b200.compress_part, on its own GPU); the ranks all-gather each
part's (bit count, CRC fold, block count); rank 0 receives the parts and
splices them at their bit offsets after the stream header on its GPU
(bzip2gpu_b200.assemble), with the end-of-stream marker and the CRC combined
from the folds (crc = rotl(crc, blocks_r) ^ fold_r).  The result is the
stream that one GPU produces for the whole input.

Collectives: one all-gather of 3 integers per rank and one point-to-point
transfer of each part to rank 0 (NCCL over NVLink for CUDA tensors, or any
backend the group uses).
"""
from __future__ import annotations


def block_ranges(n: int, block_bytes: int, world: int):
    """Byte range [a, b) of each rank: contiguous whole blocks, the block
    count split as evenly as possible (earlier ranks take the extra blocks)."""
    nb = (n + block_bytes - 1) // block_bytes
    q, r = divmod(nb, world)
    out, first = [], 0
    for k in range(world):
        cnt = q + (1 if k < r else 0)
        a = min(n, first * block_bytes)
        b = min(n, (first + cnt) * block_bytes)
        out.append((a, b))
        first += cnt
    return out


def compress_sharded(data, level: int = 9, block_bytes: int = 900000, group=None,
                     part_fn=None, assemble_fn=None):
    """Compress `data` (the whole input, present on every rank: host bytes /
    numpy array, or a CUDA tensor) with every rank of `group` taking its range
    of blocks.  Returns the stream on rank 0 and None elsewhere.

    part_fn(data_slice, block_bytes) -> (uint8 tensor, bits, fold, blocks) and
    assemble_fn(parts, bits, folds, blocks, level) -> bytes default to the
    GPU library (bzip2gpu_b200.compress_part / assemble)."""
    import torch
    import torch.distributed as dist

    if part_fn is None or assemble_fn is None:
        from . import assemble, compress_part
        part_fn = part_fn or compress_part
        assemble_fn = assemble_fn or assemble
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n = data.numel() if hasattr(data, "numel") else len(data)
    a, b = block_ranges(n, block_bytes, world)[rank]
    part, bits, fold, nblk = part_fn(data[a:b], block_bytes)
    dev = part.device
    meta = torch.tensor([bits, fold, nblk], dtype=torch.int64, device=dev)
    metas = [torch.empty_like(meta) for _ in range(world)]
    dist.all_gather(metas, meta, group=group)
    metas = [m.tolist() for m in metas]
    sizes = [((m[0] + 7) // 8 + 3) // 4 * 4 for m in metas]
    if rank == 0:
        parts = [part[: sizes[0]]]
        for r in range(1, world):
            buf = torch.empty(sizes[r], dtype=torch.uint8, device=dev)
            if sizes[r]:
                dist.recv(buf, src=dist.get_global_rank(group, r) if group else r, group=group)
            parts.append(buf)
        return assemble_fn(parts, [m[0] for m in metas], [m[1] for m in metas],
                           [m[2] for m in metas], level)
    if sizes[rank]:
        dist.send(part[: sizes[rank]].contiguous(),
                  dst=dist.get_global_rank(group, 0) if group else 0, group=group)
    return None
