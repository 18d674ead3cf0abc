"""Builds the CUDA library ``libblitz_b200.so`` for sm_100a, in place.

FP64 arithmetic of the audit must round exactly like the reference CPU build
(-ffp-contract=off): device code is compiled with --fmad=false and the host
compiler with -ffp-contract=off.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libblitz_b200.so"
SOURCES = ["topology.cu", "raster.cu", "audit.cu", "session.cu", "static_distance.cu", "surrogate.cu", "generate.cu", "mesh_io.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
    "-Xptxas", "-v",
] + os.environ.get("NVCC_EXTRA", "").split()


def needs_build() -> bool:
    if not LIB.exists():
        return True
    stamp = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "blitz_audit.h"]
    return any(d.stat().st_mtime > stamp for d in deps if d.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    objs = []
    obj_dir = HERE / "_build"
    obj_dir.mkdir(exist_ok=True)
    for src in SOURCES:
        obj = obj_dir / (Path(src).stem + ".o")
        cmd = [NVCC, *FLAGS, "-c", str(CSRC / src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src}")
        if verbose:
            sys.stderr.write(r.stderr)
        (obj_dir / (Path(src).stem + ".ptxas.txt")).write_text(r.stderr)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", str(tmp), "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
