"""Build libm3lb.so in-tree with nvcc for sm_100a.

The kernel instantiations are split over one translation unit per
(lattice, storage format) and compiled in parallel; the C ABI, the
allocation-free reduction and the serving loop are three more units.
Usage: ``python -m m3lb_b200.build [--jobs N] [--verbose]``.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libm3lb.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]

SLICES = [(lat, st) for lat in ("D2Q9", "D3Q27") for st in ("F32", "F16", "BF16", "F64", "F16C")]
HEADERS = ["lbm_common.cuh", "lbm_collide.cuh", "lbm_kernels.cuh", "lbm_stream.cuh", "lbm_rows.cuh",
           "lbm_bound.cuh",
           "lbm_launch.h",
           "lbm_host.h", "lbm_walls.h", "ctx_cache.h", "lbm_diag.cuh"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found")
    return exe


def _units():
    units = []
    for lat, st in SLICES:
        obj = BUILD / f"inst_{lat}_{st}.o"
        defs = [f"-DM3LB_LAT={lat}", f"-DM3LB_ST=k{st}", f"-DM3LB_NAME=launchers_{lat}_{st}"]
        units.append((CSRC / "lbm_inst.cu", obj, defs))
    units.append((CSRC / "lbm_capi.cu", BUILD / "capi.o", []))
    units.append((CSRC / "lbm_noalloc.cu", BUILD / "noalloc.o", []))
    units.append((CSRC / "lbm_serve.cu", BUILD / "serve.o", []))
    units.append((CSRC / "lbm_walls.cu", BUILD / "walls.o", []))
    units.append((CSRC / "lbm_scalar.cu", BUILD / "scalar.o", []))
    return units


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    deps = [src] + [CSRC / h for h in HEADERS] + [PKG.parent / "include" / "m3lb.h"]
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def up_to_date() -> bool:
    """The linked library is newer than every source and header."""
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    srcs = [CSRC / "lbm_inst.cu", CSRC / "lbm_capi.cu", CSRC / "lbm_noalloc.cu",
            CSRC / "lbm_serve.cu", CSRC / "lbm_walls.cu", CSRC / "lbm_scalar.cu",
            CSRC / "lbm_host.h",
            *[CSRC / h for h in HEADERS],
            PKG.parent / "include" / "m3lb.h"]
    return all(p.stat().st_mtime <= t for p in srcs if p.exists())


def build(jobs: int | None = None, verbose: bool = False, force: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    BUILD.mkdir(exist_ok=True)
    exe = nvcc()
    units = _units()
    todo = [u for u in units if force or _stale(u[1], u[0])]

    def compile_one(u):
        src, obj, defs = u
        cmd = [exe, *ARCH, *FLAGS, *defs, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {obj.name}:\n{r.stderr[-4000:]}")
        return obj

    if todo:
        with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            list(ex.map(compile_one, todo))
    if todo or not LIB.exists():
        cmd = [exe, *ARCH, "-shared", "-o", str(LIB), *[str(u[1]) for u in units]]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.jobs, a.verbose, a.force))
    sys.exit(0)
