"""Build libvgr_b200.so (sm_100a) in-tree with nvcc.

Usage: python build.py [--force] [--verbose]

Every .cu file in this directory is compiled for sm_100a with IEEE
floating-point semantics (no --use_fast_math: the kernels rely on explicit
round-to-nearest intrinsics and their own exp/log polynomials so that a C
restatement can reproduce them bit for bit) and linked into
../vgr_b200/_lib/libvgr_b200.so, next to the Python package that loads it.
Object files go to ../_build/ (git-ignored).  Rebuilds are incremental on
source/header modification times.
"""

from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG_ROOT = HERE.parent
LIB_DIR = PKG_ROOT / "vgr_b200" / "_lib"
BUILD_DIR = PKG_ROOT / "_build"
LIB_NAME = "libvgr_b200.so"
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "--expt-relaxed-constexpr",
    "-Xptxas",
    "-warn-spills",
]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libvgr_b200.so")
    return path


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    mtime = target.stat().st_mtime
    return any(dep.stat().st_mtime > mtime for dep in deps)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    BUILD_DIR.mkdir(parents=True, exist_ok=True)
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    sources = sorted(HERE.glob("*.cu"))
    headers = sorted(HERE.glob("*.h")) + sorted(HERE.glob("*.cuh"))
    headers += sorted((PKG_ROOT.parent / "include").glob("*.h"))
    objects: list[Path] = []
    jobs = []
    for src in sources:
        obj = BUILD_DIR / (src.stem + ".o")
        objects.append(obj)
        if force or _stale(obj, [src, *headers]):
            cmd = [nvcc(), *ARCH_FLAGS, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
            if ptxas_verbose:
                cmd[1:1] = ["-Xptxas", "-v"]
            jobs.append(cmd)

    def run(cmd: list[str]) -> subprocess.CompletedProcess:
        if verbose:
            print(" ".join(cmd), flush=True)
        return subprocess.run(cmd, capture_output=True, text=True)

    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as pool:
        for cmd, result in zip(jobs, pool.map(run, jobs)):
            if result.returncode != 0:
                sys.stderr.write(result.stdout + result.stderr)
                raise RuntimeError(f"nvcc failed for {cmd[-3]}")
            if (verbose or ptxas_verbose) and (result.stdout or result.stderr):
                sys.stderr.write(result.stdout + result.stderr)

    lib = LIB_DIR / LIB_NAME
    if force or jobs or _stale(lib, objects):
        cmd = [nvcc(), *ARCH_FLAGS, "-shared", "-o", str(lib), *map(str, objects), "-lcudart"]
        result = run(cmd)
        if result.returncode != 0:
            sys.stderr.write(result.stdout + result.stderr)
            raise RuntimeError("nvcc link of libvgr_b200.so failed")
    return lib


if __name__ == "__main__":
    parser = argparse.ArgumentParser()
    parser.add_argument("--force", action="store_true")
    parser.add_argument("--verbose", action="store_true")
    parser.add_argument("--ptxas-verbose", action="store_true")
    args = parser.parse_args()
    print(build(force=args.force, verbose=args.verbose, ptxas_verbose=args.ptxas_verbose))
