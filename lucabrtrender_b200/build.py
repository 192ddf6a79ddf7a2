"""Build the in-tree CUDA library ``lucabrtrender_b200/lib/liblrt_raster.so``.

Every kernel is compiled for sm_100a only. ``-fmad=false`` keeps each float
product and sum a separate rounding, in source order, which is what makes the
kernels' tile tests, depth keys and blend bit-identical to the CPU oracle.
The files whose results are checked to a tolerance instead (the backward
blend and the loss, CONTRACTED) are compiled with ``-fmad=true``: the
compiler may fuse a product into the sum that follows it. The per-splat
backward (train.cu) is not: its single-view and per-chunk kernels inline
the same chain rule and must give the same bits, and where the compiler
fuses is decided per kernel after inlining, which made the two differ.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
LIB_DIR = PACKAGE / "lib"
LIBRARY = LIB_DIR / "liblrt_raster.so"
OBJ_DIR = ROOT / "_build" / "obj"

SOURCES = ["project.cu", "scan.cu", "sort.cu", "blend.cu", "blend_backward.cu", "raster.cu", "math_eval.cu", "scan_noalloc.cu", "train.cu", "decode.cu", "compare.cu", "loss.cu", "lod.cu", "lod_host.cu", "train_batch.cu", "filter3d.cu", "host.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
         "-I", str(ROOT / "include")]
CONTRACTED = {"blend_backward.cu", "loss.cu"}


def fmad_flag(name: str) -> str:
    return "-fmad=true" if name in CONTRACTED else "-fmad=false"


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = Path(cuda) / "bin" / "nvcc"
    return str(path) if path.exists() else "nvcc"


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "lrt_raster.h"]


def _compile(src: Path, obj: Path, verbose_ptxas: bool) -> None:
    cmd = [nvcc(), *ARCH, *FLAGS, fmad_flag(src.name), "-c", str(src), "-o", str(obj)]
    if verbose_ptxas and src.suffix == ".cu":
        cmd += ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    if verbose_ptxas:
        sys.stderr.write(res.stderr)


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    # The headers and this file (its flags) are inputs of every object.
    newest_header = max([p.stat().st_mtime for p in _headers()] + [Path(__file__).stat().st_mtime])
    jobs = []
    objs = []
    for name in SOURCES:
        src = CSRC / name
        obj = OBJ_DIR / (name + ".o")
        objs.append(obj)
        stale = (not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header))
        if force or stale or verbose_ptxas:
            jobs.append((src, obj))
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as pool:
        for f in [pool.submit(_compile, s, o, verbose_ptxas) for s, o in jobs]:
            f.result()
    if force or jobs or not LIBRARY.exists() or LIBRARY.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = LIBRARY.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lpthread"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        tmp.replace(LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv)
    print(LIBRARY)
