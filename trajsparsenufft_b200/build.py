"""Build the in-tree C++/CUDA host library ``libtrajsparsenufft.so`` for sm_100a.

Objects go to ``trajsparsenufft_b200/_build`` (git-ignored); the shared library is
written next to this file so it travels with the source tree.  Rebuilds are
incremental on source/header modification times.

    python -m trajsparsenufft_b200.build [--verbose] [--ptxas-info]
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SRC = PKG / "csrc"
OUT = PKG / "_build"
LIB = PKG / "libtrajsparsenufft.so"

HOST_SOURCES = ["planner.cpp", "kb.cpp", "pack_io.cpp", "api_host.cpp"]
CUDA_SOURCES = ["kernels.cu", "plan.cu", "noalloc.cu", "interp_tc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found (CUDA 12.9 toolkit required)")


def _headers() -> list[Path]:
    return list(SRC.glob("*.hpp")) + list(SRC.glob("*.cuh")) + [ROOT / "include" / "trajsparsenufft.h"]


def _stale(obj: Path, src: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> Path:
    nvcc = _nvcc()
    OUT.mkdir(exist_ok=True)
    deps = _headers()
    inc = ["-I", str(ROOT / "include"), "-I", str(SRC)]
    objs = []
    jobs = []
    for name in HOST_SOURCES:
        src, obj = SRC / name, OUT / (name + ".o")
        objs.append(obj)
        if force or _stale(obj, src, deps):
            jobs.append(["g++", "-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
                         *inc, "-c", str(src), "-o", str(obj)])
    for name in CUDA_SOURCES:
        src, obj = SRC / name, OUT / (name + ".o")
        objs.append(obj)
        if force or _stale(obj, src, deps):
            cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
                   "-Xcompiler", "-fPIC,-ffp-contract=off", *inc, "-c", str(src), "-o", str(obj)]
            if ptxas_info:
                cmd[1:1] = ["-Xptxas", "-v"]
            jobs.append(cmd)
    procs = []
    for cmd in jobs:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for cmd, p in procs:
        out, _ = p.communicate()
        if out and (verbose or ptxas_info or p.returncode):
            print(out, file=sys.stderr)
        if p.returncode:
            failed.append(cmd[-3])
    if failed:
        raise RuntimeError(f"compilation failed: {failed}")
    if jobs or not LIB.exists() or force:
        link = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lpthread"]
        if verbose:
            print(" ".join(link), flush=True)
        subprocess.run(link, check=True)
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(args.verbose, args.ptxas_info, args.force))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
