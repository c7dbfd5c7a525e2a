"""Build libcudams_b200.so (sm_100a) in-tree.

Usage:  python cosine-similarity_b200/build_native.py [--ptxas-verbose] [--force]

Compiles every csrc/*.cu with nvcc for sm_100a only and links them into
cudams/libcudams_b200.so next to the Python package that loads it.  Object
files go to _build/ (git-ignored).  Incremental: a source is recompiled only
when it or a header is newer than its object.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "cudams" / "libcudams_b200.so"
INCLUDE = HERE.parent / "include"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
    # keep IEEE division / sqrt and explicit rounding: results must be
    # bit-identical to the oracle
    "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-I", str(INCLUDE),
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; cannot build libcudams_b200.so")
    return cand


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = False) -> Path:
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    headers = sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))
    newest_header = max((h.stat().st_mtime for h in headers), default=0.0)
    objs = []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        stale = (force or not obj.exists() or obj.stat().st_mtime < src.stat().st_mtime
                 or obj.stat().st_mtime < newest_header)
        if not stale:
            continue
        cmd = [nvcc, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
        if ptxas_verbose:
            cmd[1:1] = ["-Xptxas", "-v"]
        if not quiet:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    relink = force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs)
    if relink:
        cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
               *[str(o) for o in objs], "-o", str(LIB), "-cudart", "static"]
        if not quiet:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    args = ap.parse_args(argv)
    lib = build(force=args.force, ptxas_verbose=args.ptxas_verbose)
    print(f"built {lib}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
