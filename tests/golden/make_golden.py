"""Make the golden fixtures that pin the oracle to the reference.

  python tests/golden/make_golden.py testoracles
      Runs the reference's own CPU test oracles (oracle/_ref/
      libref_testoracles.so, built from the reference tree by
      `make -C oracle ref`) on the reference tests' glibc rand() vectors and
      writes their output digests to tests/golden/ref_testoracles.json.

  python tests/golden/make_golden.py inputs <dir>
      Writes the inputs of the reference GPU run to <dir> (workload bytes from
      bzip2gpu_b200.workloads; the byte streams are deterministic).

  python tests/golden/make_golden.py refdumps <dir>
      Digests the per-stage dumps that oracle/_ref/ref_harness wrote on a B200
      (one <dir>/<case>/ folder per input, plus <dir>/<case>.stream<k>.bz2
      from its `stream` mode) into tests/golden/ref_gpu.json.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import conftest as C  # noqa: E402


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def vectors():
    """Reference test vectors: name -> (stage, input, extra)."""
    v = {}
    for R in (20, 3, 10000):
        v[f"rle1_R{R}"] = ("rle1", C.ref_rle1_input(R), None)
    for A in (256, 4, 1):
        v[f"bwt_A{A}"] = ("bwt", C.ref_bwt_input(A), None)
    for A in (256, 4):
        v[f"mtf_A{A}"] = ("mtf", C.ref_mtf_input(A), None)
    for R in (20, 10000):
        a = C.ref_rle2_input(R)
        v[f"rle2_R{R}"] = ("rle2", a, C.table_size(a))
    a = C.ref_rle2_incompressible()
    v["rle2_incompressible"] = ("rle2", a, C.table_size(a))
    return v


def cmd_testoracles():
    import oracle
    R = oracle.ref_lib()
    if R is None:
        raise SystemExit("oracle/_ref/libref_testoracles.so missing: run `make -C oracle ref`")
    res = {}
    for name, (stage, a, extra) in vectors().items():
        if stage == "rle1":
            out = np.zeros(2 * a.size, np.uint8)
            m = R.ref_rle1(a.ctypes.data, a.size, out.ctypes.data)
            out = out[:m]
        elif stage == "bwt":
            out = np.zeros(a.size, np.int32)
            R.ref_bwt(a.ctypes.data, a.size, out.ctypes.data)
        elif stage == "mtf":
            out = np.zeros(a.size, np.uint8)
            R.ref_mtf_plain(a.ctypes.data, a.size, out.ctypes.data)
        else:
            out = np.zeros(2 * a.size + 1, np.uint16)
            s = R.ref_rle2(a.ctypes.data, a.size, extra, out.ctypes.data)
            out = out[:s]
        res[name] = {"stage": stage, "input_sha256": sha(a), "len": int(out.size),
                     "output_sha256": sha(out)}
        print(name, out.size)
    (HERE / "ref_testoracles.json").write_text(json.dumps(res, indent=1, sort_keys=True) + "\n")


# inputs of the reference GPU run: name -> callable returning bytes
def gpu_cases():
    import bzip2gpu_b200.workloads as W
    return {
        "cfg0_markov_4MiB": lambda: W.small_markov(),
        "zeros_2MiB": lambda: np.zeros(2 << 20, np.uint8),
        "periodic17_1MiB": lambda: W.periodic17(1 << 20),
        "uniform_300KiB": lambda: __import__("bzip2gpu_b200").gen_uniform(300 << 10, 0xB2C1C),
    }


def cmd_inputs(d: Path):
    d.mkdir(parents=True, exist_ok=True)
    for name, f in gpu_cases().items():
        if f is None:
            continue
        a = np.ascontiguousarray(f(), dtype=np.uint8)
        (d / f"{name}.bin").write_bytes(a.tobytes())
        print(name, a.size, sha(a))


def cmd_refdumps(d: Path):
    res = {}
    for case in sorted(p for p in d.iterdir() if p.is_dir()):
        blocks = []
        if not (case / "scalars.txt").exists() or not (case / "scalars.txt").read_text().strip():
            print(case.name, "incomplete (the reference run did not finish), skipped")
            continue
        sc = (case / "scalars.txt").read_text().split("\n")
        for line in sc:
            if not line.strip():
                continue
            parts = line.split()
            k = int(parts[0])
            kv = dict(p.split("=") for p in parts[1:])
            pre = case / f"b{k}"
            rec = {kk: int(vv) for kk, vv in kv.items()}
            for stage, dt in (("rle1", np.uint8), ("sa", np.int32), ("mtf", np.uint8),
                              ("present", np.uint8), ("rle2", np.uint16), ("sel", np.uint8),
                              ("payload", np.uint32)):
                a = np.fromfile(f"{pre}.{stage}", dtype=dt)
                if stage == "payload":
                    a = a[: (rec["bits"] + 31) // 32]
                rec[f"{stage}_sha256"] = sha(a)
            ln = np.fromfile(f"{pre}.len", dtype=np.uint8).reshape(6, 258)
            code = np.fromfile(f"{pre}.code", dtype=np.int32).reshape(6, 258)
            alpha = rec["n_in_use"] + 2
            ng = rec["n_groups"]
            rec["len_sha256"] = sha(ln[:ng, :alpha])
            rec["code_sha256"] = sha(code[:ng, :alpha])
            blocks.append(rec)
        streams = {}
        for sp in sorted(d.glob(f"{case.name}.stream*.bz2")):
            b = sp.read_bytes()
            streams[sp.name] = {"len": len(b), "sha256": hashlib.sha256(b).hexdigest()}
        res[case.name] = {"blocks": blocks, "streams": streams}
        print(case.name, len(blocks), streams)
    (HERE / "ref_gpu.json").write_text(json.dumps(res, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    cmd = sys.argv[1] if len(sys.argv) > 1 else "testoracles"
    if cmd == "testoracles":
        cmd_testoracles()
    elif cmd == "inputs":
        cmd_inputs(Path(sys.argv[2]))
    elif cmd == "refdumps":
        cmd_refdumps(Path(sys.argv[2]))
    else:
        raise SystemExit(__doc__)
