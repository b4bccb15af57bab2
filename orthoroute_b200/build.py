"""Builds liborsp.so (the sm_100a CUDA kernels behind the C ABI in include/orsp.h).

The library is compiled in-tree with nvcc so that it travels with the source
tree; there is no JIT step at import time.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
REPO_DIR = PKG_DIR.parent
CSRC = PKG_DIR / "csrc"
INCLUDE = REPO_DIR / "include"
LIB_PATH = PKG_DIR / "liborsp.so"

SOURCES = [
    "orsp_graph.cu",
    "orsp_sssp.cu",
    "orsp_batch.cu",
    "orsp_accounting.cu",
    "orsp_roi.cu",
    "orsp_lattice.cu",
    "orsp_via.cu",
    "orsp_route.cu",
    "orsp_warm.cu",
    "orsp_warm_tc.cu",
    "orsp_bookkeeping.cu",
    "orsp_geometry.cu",
]

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; liborsp.so cannot be built")
    return cand


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build_library(force: bool = False, verbose: bool = False, extra_flags=None) -> Path:
    """Compiles every .cu source into liborsp.so (skips work when up to date)."""
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [INCLUDE / "orsp.h"]
    if not force and not _stale(LIB_PATH, deps):
        return LIB_PATH
    build_dir = PKG_DIR / "_build"
    build_dir.mkdir(exist_ok=True)
    nvcc = nvcc_path()
    common = [
        "-O3",
        "-lineinfo",
        "-std=c++17",
        "-Xcompiler",
        "-fPIC",
        "-Xcompiler",
        "-fvisibility=hidden",
        f"-I{INCLUDE}",
        f"-I{CSRC}",
        *ARCH_FLAGS,
    ]
    if extra_flags:
        common += list(extra_flags)
    objs = []
    for src in SOURCES:
        obj = build_dir / (Path(src).stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [CSRC / src, INCLUDE / "orsp.h", *CSRC.glob("*.cuh")]):
            cmd = [nvcc, *common, "-c", str(CSRC / src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH_FLAGS, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True)
    print(LIB_PATH)
