"""Builds the native libraries of helio_b200 in-tree.

* ``helio_b200/lib/libhelio_cull.so`` — the CUDA kernels (sm_100a) and the C-ABI of
  ``include/helio_cull.h``;
* ``helio_b200/lib/libhelio_scenegen.so`` — the seeded synthetic-input generator (host only).

Usage: ``python -m helio_b200.build`` (or ``build()`` from Python). Object files
go to ``helio_b200/_build``; rebuilds are incremental on source timestamps.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
OBJ = PKG / "_build"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")

CUDA_SOURCES = ["capi.cu", "hiz.cu", "instance_cull.cu", "vg_cull.cu", "noalloc.cu", "batch.cu", "batch_api.cu", "serve.cu", "vg_build.cu", "shadow_cull.cu"]
HEADERS = ["common.cuh", "tma.cuh", "kernels.h", "vg.h", "instance_cull.h", "hiz_tile.cuh", "vg_device.cuh", "host_util.h", "batch.h",
           "shadow_device.cuh", "shadow_host.h"]

# IEEE binary32 without contraction, correctly rounded division / square root,
# denormals preserved: visibility and LOD decisions must be bit-reproducible.
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    f"-I{ROOT / 'include'}",
]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build failed: {' '.join(cmd)}")


def build_cuda(verbose_ptxas: bool = False) -> Path:
    LIB.mkdir(exist_ok=True)
    OBJ.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [ROOT / "include" / "helio_cull.h"]
    jobs = []
    objs = []
    for src in CUDA_SOURCES:
        s = CSRC / src
        o = OBJ / (src + ".o")
        objs.append(o)
        if _stale(o, [s, *headers]) or verbose_ptxas:
            extra = ["-Xptxas", "-v"] if verbose_ptxas else []
            jobs.append([NVCC, *NVCC_FLAGS, *extra, "-c", str(s), "-o", str(o)])
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(_run, jobs))
    out = LIB / "libhelio_cull.so"
    if _stale(out, objs):
        _run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(out),
              *map(str, objs), "-lcudart_static", "-lrt", "-lpthread", "-ldl"])
    return out


def build_scenegen() -> Path:
    LIB.mkdir(exist_ok=True)
    src = CSRC / "scenegen.cpp"
    out = LIB / "libhelio_scenegen.so"
    if _stale(out, [src, ROOT / "include" / "helio_cull.h"]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", str(src), "-o", str(out)])
    return out


def build_all() -> list[Path]:
    return [build_cuda(), build_scenegen()]


if __name__ == "__main__":
    v = "--ptxas" in sys.argv
    print(build_cuda(verbose_ptxas=v))
    print(build_scenegen())
