"""Benchmark: bzip2 compression throughput on B200 (plain form).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--size BYTES] [--impl ours|reference]

Workload: the large Markov stream (order-1 Markov bytes, alphabet and
Dirichlet concentration redrawn every 64 MiB, 2 % run starts of length
4..300, 900,000-byte blocks, seed 0xB2C4), generated on the device.  A step
compresses the whole stream to a complete .bz2 stream.
  value  MB/s of input, input resident in HBM when the timed region starts,
         the complete stream delivered to a page-locked host buffer
         (bz2g_compress_device_into).
  e2e    MB/s through bz2g_compress_into with input and output in page-locked
         host memory: the host->device copy of every input byte and the
         device->host copy of the stream are inside the timed region.
After the timed regions (unless --no-check): the whole plain stream is
compared byte for byte with the oracle's stream of the same input, and the
whole learned-form and bzip2-format streams are decoded by libbz2 (every
block) and compared with the input ("checks" in the JSON line).
Under torchrun each rank compresses its own stream (weak scaling, no
collective on the data path); times are the max over ranks.
--impl reference times the reference path's CPU implementation (the oracle
port of the reference semantics; the reference itself has no CPU compressor)
on a bounded sample of the same workload with all host threads.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "MB/s compressed on 1 B200: plain vs batched+learned at equal ratio; %HBM peak"
WORKLOAD = "large Markov stream, 900k blocks (order-1 Markov, alphabet/alpha redrawn every 64 MiB, 2% runs)"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[1]) for s in self.samples if len(s) > 2 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 2 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_sample_time(host, threads: int):
    import oracle
    t = time.perf_counter()
    out = oracle.compress(host, 9, 900000, threads=threads)
    return time.perf_counter() - t, len(out)


CPU_SAMPLE_NOTE = ("the first 1,800,000 bytes (two blocks) of each of the stream's 64 MiB "
                   "segments, so every parameter redraw is in the sample")


def run_reference(args):
    """The reference path on the host cores (the oracle port of its
    semantics), on a bounded sample of the same stream.  Nothing of the
    product library is loaded: the sample comes from the oracle's generator,
    whose bytes a CPU test pins to the product generator's."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    threads = os.cpu_count() or 1
    host = oracle.large_stream_sample(args.size)
    sample = host.size
    for _ in range(args.warmup):
        cpu_sample_time(host[: 8 << 20], threads)
    times = []
    for _ in range(args.steps):
        dt, _ = cpu_sample_time(host, threads)
        times.append(dt)
    tot = sum(times)
    mbps = sample * len(times) / tot / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(mbps, 2), "unit": "MB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(tot / len(times) * 1e3, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": WORKLOAD, "bytes_per_rank": args.size, "sample_bytes": sample,
                   "block_bytes": 900000, "level": 9},
        "cpu_baseline": {"value": round(mbps, 2), "unit": "MB/s", "cores": threads,
                         "kind": "port",
                         "sample": f"{sample} bytes: {CPU_SAMPLE_NOTE}; {threads} threads, "
                                   f"one block per thread"},
        "e2e": {"value": round(mbps, 2), "unit": "MB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def many_inputs(B, W, torch, rank: int, world: int, count: int, plain_steps: int,
                batched_steps: int, warmup: int) -> dict:
    """Batched form vs plain form on the many-inputs workload: inputs of
    log-uniform size 1 KiB .. 8 MiB, alphabet 2..256, alpha 0.05 .. 5, level
    1..9 (blocks of level * 100,000 bytes), 1 % runs; inputs resident in HBM,
    streams delivered to page-locked host memory.  "plain" compresses the
    inputs one call each; "batched" runs all their blocks through shared slabs
    in one call (slab shapes from the committed tuning table).  The batched
    streams are checked to be the per-input streams, byte for byte."""
    items = W.batch_inputs(count=count, seed=0xB2C2 + 7919 * rank)
    sizes = [x.data.size for x in items]
    levels = [x.level for x in items]
    total = sum(sizes)
    flat = torch.from_numpy(np.concatenate([x.data for x in items])).cuda()
    del items
    offs = np.concatenate([[0], np.cumsum(sizes)])
    d_in = [flat[offs[i]:offs[i + 1]] for i in range(len(sizes))]
    cap = B.lib().bz2g_compress_batch_bound(len(sizes), (ctypes.c_size_t * len(sizes))(*sizes),
                                           (ctypes.c_int * len(sizes))(*levels), None)
    h_out = torch.empty(cap, dtype=torch.uint8, pin_memory=True)

    def plain():
        n = 0
        for x, lv in zip(d_in, levels):
            n += B.compress_device_into(x, h_out[n:], lv, lv * 100000)
        return n

    def batched():
        st = B.compress_batch(d_in, levels, out=h_out, on_device=True)
        return sum(len(v) for v in st)

    ref = [bytes(v) for v in B.compress_batch(d_in, levels, on_device=True)]
    for _ in range(warmup):
        plain()
        batched()
    res = {}
    for name, fn, steps in (("plain", plain, plain_steps), ("batched", batched, batched_steps)):
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            nbytes = fn()
        e1.record()
        torch.cuda.synchronize()
        dt = max_over_ranks(e0.elapsed_time(e1) / 1e3, world)
        res[name] = {"MB/s": round(total * world * steps / dt / 1e6, 2), "timed_passes": steps,
                     "ms_per_pass": round(dt / steps * 1e3, 2), "stream_bytes": int(nbytes)}
    # the batched streams are the per-input streams
    exact = True
    for i, (x, lv) in enumerate(zip(d_in, levels)):
        k = B.compress_device_into(x, h_out, lv, lv * 100000)
        exact = exact and bytes(h_out[:k].numpy()) == ref[i]
    del d_in, flat, h_out
    torch.cuda.empty_cache()
    return {"workload": "many inputs (1 KiB..8 MiB; levels 1..9)", "inputs": len(sizes),
            "bytes": int(total), "forms": res,
            "batched_over_plain": round(res["batched"]["MB/s"] / res["plain"]["MB/s"], 3),
            "bit_exact": bool(exact)}


def run_batch(args):
    """The many-inputs workload alone (see many_inputs)."""
    world, rank, local = dist_setup(args.gpus)
    import torch

    import bzip2gpu_b200 as B
    import bzip2gpu_b200.workloads as W
    B.set_timing(False)
    res = many_inputs(B, W, torch, rank, world, args.batch_count, args.steps, args.steps,
                      args.warmup)
    if rank == 0:
        res.update({"n_gpus": world, "steps": args.steps, "warmup": args.warmup})
        print(json.dumps(res))


def run_stress(args):
    """The BWT stress stream (zeros | periodic-17 | uniform | Markov, 64 MiB
    each, 900,000-byte blocks): MB/s, the stream checked against the oracle,
    and the BWT's HBM GB/s per doubling round by the byte model (28 bytes per
    rotation still in a group of two or more, over the round's device time).
    One worker stream by default, so each round's time is its own."""
    world, rank, local = dist_setup(args.gpus)
    import torch

    import bzip2gpu_b200 as B
    import bzip2gpu_b200.workloads as W
    import oracle

    host = W.stress()
    d_in = torch.from_numpy(host).cuda()
    B.set_engine(args.slab or 128, args.workers or 1)
    B.set_timing(True)
    out = B.compress_device(d_in, 9)
    for _ in range(max(args.warmup - 1, 0)):
        B.compress_device(d_in, 9)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        got = B.compress_device(d_in, 9)
    e1.record()
    torch.cuda.synchronize()
    dt = e0.elapsed_time(e1) / 1e3
    rounds = B.last_round_stats()
    stats = B.last_stats()
    peak, peak_kind = peaks()
    rows = []
    for r in rounds:
        shift = None if r["round"] == 0 else 4 << (r["round"] - 1)
        gbs = 28 * r["active"] / (r["ms"] / 1e3) / 1e9 if r["ms"] > 0 else 0.0
        rows.append({"round": r["round"], "shift": shift, "active": r["active"],
                     "ms": round(r["ms"], 3), "model_GBps": round(gbs, 1),
                     "frac_of_hbm": round(gbs / peak, 4)})
    identical = got == out and out == oracle.compress(host, 9, threads=os.cpu_count() or 8)
    if rank == 0:
        print(json.dumps({"workload": "BWT stress: zeros | periodic-17 | uniform | Markov, "
                                      "64 MiB each, 900k blocks", "bytes": int(host.size),
                          "MB/s": round(host.size * args.steps / dt / 1e6, 2),
                          "identical_to_oracle": bool(identical), "workers": args.workers or 1,
                          "peak_GBps": peak, "peak_kind": peak_kind,
                          "stage_ms": {k[3:]: round(v, 2) for k, v in stats.items()
                                       if k.startswith("ms_")},
                          "bwt_rounds": rows}))


# DRAM bytes per algorithmic byte of k_radix_scatter: (255.06 + 203.20) MB /
# 494.13 MB in an ncu capture of the second pass of the first sort over a
# 128-block slab (profiles/k_radix_scatter_ncu_full_256MiB.md)
TRAFFIC_PER_ALGO_BYTE = (255.06 + 203.20) / 494.13


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--size", type=int, default=10 << 30)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-isolated", action="store_true",
                    help="skip the one-worker timing of the scatter kernel")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the many-inputs (batched form) measurement")
    ap.add_argument("--no-check", action="store_true",
                    help="skip the whole-stream parity and round-trip checks")
    ap.add_argument("--slab", type=int, default=0)
    ap.add_argument("--workers", type=int, default=0)
    ap.add_argument("--workload", default="large", choices=["large", "batch", "stress"])
    ap.add_argument("--batch-count", type=int, default=2048)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "stress":
        return run_stress(args)

    world, rank, local = dist_setup(args.gpus)
    import torch

    import bzip2gpu_b200 as B
    import bzip2gpu_b200.workloads as W

    if args.slab or args.workers:
        B.set_engine(args.slab, args.workers)
    n = args.size
    seed = 0xB2C4 + 7919 * rank
    d_in = W.large_stream(n, seed=seed, device=True)
    torch.cuda.synchronize()
    B.set_timing(True)

    # warm-up; the first stream is kept to check the timed ones against it
    out = B.compress_device(d_in, 9)
    ratio = len(out) / n
    h_out = torch.empty(int(len(out) * 1.25) + (1 << 20), dtype=torch.uint8, pin_memory=True)
    for _ in range(max(args.warmup - 1, 0)):
        B.compress_device_into(d_in, h_out, 9)

    def timed(fn):
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        res = None
        for _ in range(args.steps):
            res = fn()
        e1.record()
        torch.cuda.synchronize()
        barrier(world)
        return e0.elapsed_time(e1) / 1e3, res

    l0 = B.launch_count()
    with Clocks(local) as clk:
        dt, olen = timed(lambda: B.compress_device_into(d_in, h_out, 9))
    assert olen == len(out) and bytes(h_out[:olen].numpy()) == out
    launches = (B.launch_count() - l0) // max(args.steps, 1)
    stats = B.last_stats()
    # the batched form on the same stream (one input: blocks in one queue),
    # warmed like the plain form
    for _ in range(args.warmup):
        B.compress_batch([d_in], [9], [900000], out=h_out, on_device=True)
    bt, bout = timed(lambda: B.compress_batch([d_in], [9], [900000], out=h_out, on_device=True))
    assert bytes(bout[0]) == out
    bt = max_over_ranks(bt, world)
    batched_value = n * world * args.steps / bt / 1e6
    # batched + learned selector (shipped parameters); the streams differ
    # from the reference's, so they are checked by decoding, and their size
    # is reported against the plain stream's
    learned = None
    import bzip2gpu_b200.selector as SEL
    if SEL.WEIGHTS.exists():
        SEL.load_default()
        B.set_selector("learned")
        try:
            for _ in range(args.warmup):
                B.compress_batch([d_in], [9], [900000], out=h_out, on_device=True)
            lt, lout = timed(lambda: B.compress_batch([d_in], [9], [900000], out=h_out,
                                                      on_device=True))
            lbytes = bytes(lout[0])
        finally:
            B.set_selector("plain")
        lt = max_over_ranks(lt, world)
        learned = {"MB/s": round(n * world * args.steps / lt / 1e6, 2),
                   "ratio": round(len(lbytes) / n, 5),
                   "size_vs_plain": round(len(lbytes) / len(out), 6)}
    # bzip2 1.0.8's block format (block split by RLE1 length, 255-byte runs;
    # byte-identical to libbz2), split included; checked by decoding a prefix
    for _ in range(args.warmup):
        B.compress_device_into(d_in, h_out, 9, B.BZIP2_BLOCKS)
    zt, zlen = timed(lambda: B.compress_device_into(d_in, h_out, 9, B.BZIP2_BLOCKS))
    zbytes = bytes(h_out[:zlen].numpy())
    zt = max_over_ranks(zt, world)
    bzip2_form = {"MB/s": round(n * world * args.steps / zt / 1e6, 2),
                  "ratio": round(zlen / n, 5), "size_vs_plain": round(zlen / len(out), 6)}
    dt = max_over_ranks(dt, world)
    value = n * world * args.steps / dt / 1e6

    # the many-inputs workload: per-input plain calls vs the batched form
    batch_many = None
    if not args.no_batch:
        B.set_timing(False)
        batch_many = many_inputs(B, W, torch, rank, world, args.batch_count, 1, 3, 1)
        B.set_timing(True)

    e2e = None
    decode = None
    if not args.no_e2e:
        h_in = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        h_in.copy_(d_in)
        del d_in
        torch.cuda.synchronize()
        B.compress_into(h_in, h_out, 9)  # warm the host path
        dte, oute = timed(lambda: B.compress_into(h_in, h_out, 9))
        assert oute == len(out) and bytes(h_out[:oute].numpy()) == out
        # the GPU decoder on the same stream (every block CRC and the stream
        # CRC are checked by the decoder): device-resident (stream and output
        # in HBM) and end to end (pinned host stream in, pinned host bytes out)
        h_comp = torch.empty(len(out), dtype=torch.uint8, pin_memory=True)
        h_comp.numpy()[:] = np.frombuffer(out, np.uint8)
        d_comp = h_comp.cuda()
        d_dec = torch.empty(n, dtype=torch.uint8, device="cuda")
        B.decompress_into(d_comp, d_dec)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        assert B.decompress_into(d_comp, d_dec) == n
        torch.cuda.synchronize()
        ddt = max_over_ranks(time.perf_counter() - t0, world)
        same = all(torch.equal(d_dec[i:i + (1 << 30)], h_in[i:i + (1 << 30)].cuda())
                   for i in range(0, n, 1 << 30))
        del d_dec, d_comp
        h_dec = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        t0 = time.perf_counter()
        assert B.decompress_into(h_comp, h_dec) == n
        hdt = max_over_ranks(time.perf_counter() - t0, world)
        same = same and torch.equal(h_dec[-(1 << 24):], h_in[-(1 << 24):]) and \
            torch.equal(h_dec[: 1 << 24], h_in[: 1 << 24])
        del h_dec, h_comp
        decode = {"MB/s": round(n * world / ddt / 1e6, 2), "unit": "MB/s of output",
                  "api": "bz2g_decompress_device_into (stream and output in HBM)",
                  "e2e_MB/s": round(n * world / hdt / 1e6, 2),
                  "e2e_api": "bz2g_decompress_into (pinned host stream in, pinned host out)",
                  "output_identical": bool(same)}
        dte = max_over_ranks(dte, world)
        e2e = {"value": round(n * world * args.steps / dte / 1e6, 2), "unit": "MB/s",
               "h2d_bytes_per_step": n, "d2h_bytes_per_step": int(oute),
               "api": "bz2g_compress_into (pinned host input and output)"}
        host = h_in.numpy()
    else:
        host = d_in.cpu().numpy()

    # Whole-stream checks (outside the timed regions): the plain stream equals
    # the oracle's stream of the same input byte for byte, and the learned and
    # bzip2-format streams decode to the input through libbz2, every block
    # (each re-wrapped as a stream of its own, decoded on all host threads);
    # the learned stream also through this library's GPU decoder.
    checks = None
    if not args.no_check:
        import oracle
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        identical = oracle.compress(host, 9, 900000, threads=threads) == out
        checks = {"parity": {"bytes": n, "stream_bytes": len(out), "identical": bool(identical),
                             "against": f"oracle port of the reference path, {threads} threads",
                             "seconds": round(time.perf_counter() - t0, 1)}}
        if learned is not None:
            rt = oracle.libbz2_matches(lbytes, host, threads)
            dec = memoryview(B.decompress(lbytes))
            rt["gpu_decoder_identical"] = len(dec) == n and all(
                dec[i:i + (1 << 28)] == host[i:i + (1 << 28)].tobytes()
                for i in range(0, n, 1 << 28))
            del dec
            learned["round_trip"] = bool(rt["identical"] and rt["gpu_decoder_identical"])
            checks["learned_round_trip"] = rt
        rt = oracle.libbz2_matches(zbytes, host, threads)
        bzip2_form["round_trip"] = bool(rt["identical"])
        checks["bzip2_format_round_trip"] = rt

    peak, peak_kind = peaks()
    mb = B.model_bytes(stats)
    step_s = dt / args.steps
    # dominant kernel: the radix scatter of the BWT sort; its algorithmic
    # bytes are each sorted item read once and written once (16 B for a packed
    # 64-bit item, 24 B for a 64-bit key + 32-bit rotation), over the CUDA-event
    # durations of its launches on their worker streams in the last timed step
    sc_ms = stats["scatter_ms"]
    sc_gbs = stats["scatter_bytes"] / (sc_ms / 1e3) / 1e9 if sc_ms > 0 else 0.0
    # DRAM traffic per launch, scaled from one ncu capture of the scatter
    # (profiles/k_radix_scatter_ncu_full_256MiB.md: 0.927 DRAM bytes per
    # algorithmic byte) by this launch's algorithmic bytes
    per_launch = stats["scatter_bytes"] / max(stats["scatter_launches"], 1)
    traffic = int(per_launch * TRAFFIC_PER_ALGO_BYTE)
    roof = {"bound": "hbm", "achieved": round(sc_gbs, 1), "peak": peak, "unit": "GB/s",
            "frac": round(sc_gbs / peak, 4), "traffic": traffic,
            "traffic_source": "ncu dram bytes of a first-sort scatter pass (256 MiB stream, "
                              "128-block slab), 0.927 per algorithmic byte, scaled to this launch",
            "kernel": "k_radix_scatter (BWT radix sort scatter)",
            "launches_per_step": int(stats["scatter_launches"]),
            "avg_launch_us": round(1e3 * sc_ms / max(stats["scatter_launches"], 1), 1),
            "bytes_per_launch": int(stats["scatter_bytes"] / max(stats["scatter_launches"], 1)),
            "peak_kind": peak_kind}
    pipeline = {"model_bytes_per_step": int(mb),
                "model": "n + 10m + 28A + 14s + 5g + bits/8",
                "achieved_gbs": round(mb / step_s / 1e9, 1),
                "frac_of_hbm": round(mb / step_s / 1e9 / peak, 4)}

    # The same scatter kernel with the GPU to itself: one worker stream over
    # the first 2 GiB of the stream (in the timed region above the worker
    # streams share the GPU, so each launch's event time includes the other
    # streams' kernels).  Outside the timed region; an explanation of the
    # roofline figure, not the metric.
    iso = None
    if not args.no_isolated:
        k = min(n, 2 << 30)
        d_part = h_in[:k].cuda() if not args.no_e2e else d_in[:k]
        shape = B.get_engine()
        B.set_engine(shape[0], 1)
        B.compress_device(d_part, 9)
        B.compress_device(d_part, 9)
        torch.cuda.synchronize()
        st1 = B.last_stats()
        B.set_engine(*shape)
        del d_part
        if st1["scatter_ms"] > 0:
            g1 = st1["scatter_bytes"] / (st1["scatter_ms"] / 1e3) / 1e9
            iso = {"achieved": round(g1, 1), "frac": round(g1 / peak, 4), "workers": 1,
                   "bytes": int(k), "launches": int(st1["scatter_launches"]),
                   "avg_launch_us": round(1e3 * st1["scatter_ms"] /
                                          max(st1["scatter_launches"], 1), 1)}

    cpu = None
    if rank == 0 and world == 1:
        import oracle
        threads = os.cpu_count() or 1
        sample = oracle.large_stream_sample(n, seed=seed)
        cpu_dt, _ = cpu_sample_time(sample, threads)
        cpu = {"value": round(sample.size / cpu_dt / 1e6, 2), "unit": "MB/s", "cores": threads,
               "kind": "port",
               "sample": f"{sample.size} bytes: {CPU_SAMPLE_NOTE}; oracle port of the "
                         f"reference path, {threads} threads"}
        # A familiar yardstick, not bit-comparable: bzip2 -9 (libbz2 1.0.8, through
        # Python's bz2 module, which releases the GIL) on independent 900,000-byte
        # pieces of the same sample, one piece per task on all host threads.
        import bz2
        from concurrent.futures import ThreadPoolExecutor
        pieces = [sample[i:i + 900000].tobytes() for i in range(0, sample.size, 900000)]
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            zbytes = sum(len(z) for z in ex.map(lambda x: bz2.compress(x, 9), pieces))
        zdt = time.perf_counter() - t0
        cpu["libbz2_yardstick"] = {"MB/s": round(sample.size / zdt / 1e6, 2), "threads": threads,
                                   "ratio": round(zbytes / sample.size, 4),
                                   "what": "bzip2 -9 (libbz2 1.0.8) on independent 900,000-byte "
                                           "pieces of the same sample"}

    if rank == 0:
        stage_ms = {k[3:]: round(v / args.steps if False else v, 1)
                    for k, v in stats.items() if k.startswith("ms_")}
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "MB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(step_s * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator, device-generated)",
            "config": {"workload": WORKLOAD, "bytes_per_rank": n, "block_bytes": 900000,
                       "level": 9, "form": "plain", "l2": "input larger than L2",
                       "blocks": int(stats["blocks"]), "ratio": round(ratio, 4)},
            "e2e": e2e, "roofline": roof, "roofline_isolated": iso,
            "pipeline_roofline": pipeline, "cpu_baseline": cpu,
            "forms": {"plain": round(value, 2), "batched": round(batched_value, 2),
                      "learned": learned, "bzip2_format": bzip2_form,
                      "batched_many_inputs": batch_many},
            "decode": decode, "checks": checks,
            "clocks": clk.summary(), "gpu_launches": int(launches),
            "stats": {k: stats[k] for k in ("n", "m", "A", "s", "g", "bits")},
            "stage_ms_sum_over_slabs_last_step": stage_ms,
        }
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
