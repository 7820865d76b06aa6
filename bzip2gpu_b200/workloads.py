"""Seeded synthetic workloads (the reference measures on no public data set).

Every byte comes from bzip2gpu_b200.gen_markov / gen_uniform (definition in
bzip2gpu_b200/csrc/gen.cu); per-segment parameters come from numpy's PCG64
with the seeds below.

  small_markov  config 0: 4 MiB, 96 printable symbols 0x20..0x7F,
                alpha 0.3, run starts 2 %, run length 4..300, seed 0xB2C0
  stress        config 1: four 64 MiB segments: zeros; a 17-byte string
                with no 4 equal consecutive bytes (cyclically) tiled; uniform
                bytes; the config-0 source
  batch_inputs  config 2: 2,048 inputs, sizes log-uniform 1 KiB .. 8 MiB,
                alphabet size 2..256 (random subset), alpha log-uniform
                0.05 .. 5, level 1..9 (block = level * 100,000), run starts 1 %,
                run length 4..255
  selector_specs config 3: config-2 inputs until 20,000 blocks (seed
                0xB2C3 training, 0xB2C3F held out), for the learned selector
  large_stream  config 4: 10 GiB; every 64 MiB a new alphabet (size 2..256)
                and alpha (log-uniform 0.05 .. 5); run starts 2 %, run length
                4..300, seed 0xB2C4
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import gen_markov, gen_uniform

PRINTABLE = np.arange(0x20, 0x80, dtype=np.uint8)
SEG = 64 << 20


def small_markov(n: int = 4 << 20, seed: int = 0xB2C0, device: bool = False, out=None):
    """Config-0 source (also the config-1 (d) segment with its own seed)."""
    return gen_markov(n, seed, PRINTABLE, 0.3, 0.02, 4, 300, out=out, device=device)


def periodic17(n: int, seed: int = 0xB2C1B) -> np.ndarray:
    rng = np.random.default_rng(seed)
    while True:
        p = rng.integers(0, 256, 17, dtype=np.uint8)
        q = np.concatenate([p, p[:3]])
        runs4 = any(q[i] == q[i + 1] == q[i + 2] == q[i + 3] for i in range(17))
        if not runs4:
            break
    reps = n // 17 + 1
    return np.tile(p, reps)[:n]


def stress(seg: int = SEG, device: bool = False):
    """Config 1: zeros | periodic-17 | uniform | Markov, each `seg` bytes."""
    parts = [np.zeros(seg, np.uint8), periodic17(seg), gen_uniform(seg, 0xB2C1C),
             small_markov(seg, 0xB2C1D)]
    a = np.concatenate(parts)
    if device:
        import torch
        return torch.from_numpy(a).cuda()
    return a


@dataclass
class Segment:
    seed: int
    alphabet: np.ndarray
    alpha: float


def _draw_segment(rng: np.random.Generator, seed: int) -> Segment:
    A = int(rng.integers(2, 257))
    alph = np.sort(rng.choice(256, A, replace=False)).astype(np.uint8)
    alpha = float(math.exp(rng.uniform(math.log(0.05), math.log(5.0))))
    return Segment(seed, alph, alpha)


def large_stream(n: int = 10 << 30, seed: int = 0xB2C4, out=None, device: bool = True):
    """Config 4: n bytes, parameters redrawn every 64 MiB."""
    rng = np.random.default_rng(seed)
    if out is None:
        if device:
            import torch
            out = torch.empty(n, dtype=torch.uint8, device="cuda")
        else:
            out = np.empty(n, np.uint8)
    for k in range((n + SEG - 1) // SEG):
        sg = _draw_segment(rng, seed * 1000003 + k)
        a, b = k * SEG, min(n, (k + 1) * SEG)
        gen_markov(b - a, sg.seed, sg.alphabet, sg.alpha, 0.02, 4, 300, out=out[a:b])
    return out


@dataclass
class BatchInput:
    data: np.ndarray
    level: int


@dataclass
class BatchSpec:
    size: int
    segment: Segment
    level: int

    def make(self, device: bool = False):
        sg = self.segment
        return gen_markov(self.size, sg.seed, sg.alphabet, sg.alpha, 0.01, 4, 255, device=device)


def batch_specs(count: int = 2048, seed: int = 0xB2C2, max_size: int = 8 << 20):
    """Parameters of the config-2 inputs (sizes, sources, levels), no bytes."""
    rng = np.random.default_rng(seed)
    res = []
    for i in range(count):
        size = int(math.floor(math.exp(rng.uniform(math.log(1024), math.log(max_size)))))
        sg = _draw_segment(rng, seed * 1000003 + i)
        level = int(rng.integers(1, 10))
        res.append(BatchSpec(size, sg, level))
    return res


def batch_inputs(count: int = 2048, seed: int = 0xB2C2, max_size: int = 8 << 20):
    """Config 2 inputs (host arrays) with their levels."""
    return [BatchInput(sp.make(), sp.level) for sp in batch_specs(count, seed, max_size)]


def selector_specs(blocks: int = 20000, seed: int = 0xB2C3):
    """Config 3: config-2 inputs (seed 0xB2C3 training, 0xB2C3F held out) until
    their blocks (level * 100,000 bytes each) number at least `blocks`."""
    rng = np.random.default_rng(seed)
    res, nb, i = [], 0, 0
    while nb < blocks:
        size = int(math.floor(math.exp(rng.uniform(math.log(1024), math.log(8 << 20)))))
        sg = _draw_segment(rng, seed * 1000003 + i)
        level = int(rng.integers(1, 10))
        res.append(BatchSpec(size, sg, level))
        nb += -(-size // (level * 100000))
        i += 1
    return res
