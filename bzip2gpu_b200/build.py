"""In-tree build of the bzip2gpu-b200 native library, drop-in lib and CLI.

    python -m bzip2gpu_b200.build        (or bzip2gpu_b200.build.build())

Products (all sm_100a, written under bzip2gpu_b200/_lib):
  libbz2gpu_b200.so      C-ABI (include/bz2g.h) and the C++ drop-in API
                         (include/compression.h, io.h, cli.h, crc32.h)
  libbz2gpu_b200.a       the same objects as a static archive, for programs
                         linked the way the reference links its core library
                         (one CUDA runtime in the program, so client code can
                         launch the exported count_frequencies kernel itself)
  bzip2gpu               the command line tool (same flags as the reference)
Objects go to bzip2gpu_b200/_build.  A source is recompiled when it or any
header in csrc/ or include/ is newer than its object.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INC = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "_lib"
LIBNAME = "libbz2gpu_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
           "--expt-relaxed-constexpr", f"-I{INC}", f"-I{CSRC}"] + ARCH

LIB_SOURCES = ["engine.cu", "rle1.cu", "bwt.cu", "mtf.cu", "rle2.cu", "huffman.cu", "pack.cu",
               "compressor.cu", "capi.cu", "compat.cu", "gen.cu", "noalloc.cu", "mlp.cu", "stream.cu", "decode.cu",
               "split.cu"]
CLI_SOURCES = ["cli_main.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INC.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, obj: Path, hmt: float) -> str | None:
    if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hmt):
        return None
    cmd = [_nvcc(), *NVFLAGS, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [_nvcc(), *NVFLAGS, "-x", "cu", "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src.name}\n{r.stdout}\n{r.stderr}")
    return src.name


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    hmt = _headers_mtime()
    srcs = [CSRC / s for s in LIB_SOURCES + CLI_SOURCES]
    objs = {s: BUILD / (s.stem + ".o") for s in srcs}
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        done = list(ex.map(lambda s: _compile(s, objs[s], hmt), srcs))
    if verbose:
        print("compiled:", [d for d in done if d])
    lib = LIB / LIBNAME
    lib_objs = [objs[CSRC / s] for s in LIB_SOURCES]
    if not lib.exists() or lib.stat().st_mtime < max(o.stat().st_mtime for o in lib_objs):
        tmp = lib.with_suffix(".so.tmp")
        cmd = [_nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, lib_objs), "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, lib)
    arch = LIB / "libbz2gpu_b200.a"
    if not arch.exists() or arch.stat().st_mtime < max(o.stat().st_mtime for o in lib_objs):
        tmp = arch.with_suffix(".a.tmp")
        if tmp.exists():
            tmp.unlink()
        r = subprocess.run(["ar", "rcs", str(tmp), *map(str, lib_objs)], capture_output=True,
                           text=True)
        if r.returncode != 0:
            raise RuntimeError(f"archive failed\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, arch)
    cli = LIB / "bzip2gpu"
    cli_obj = objs[CSRC / "cli_main.cpp"]
    if not cli.exists() or cli.stat().st_mtime < max(lib.stat().st_mtime, cli_obj.stat().st_mtime):
        cmd = [_nvcc(), *ARCH, "-o", str(cli), str(cli_obj), f"-L{LIB}", "-lbz2gpu_b200",
               "-Xlinker", "-rpath,$ORIGIN", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"cli link failed\n{r.stdout}\n{r.stderr}")
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
