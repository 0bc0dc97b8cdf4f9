"""Build ``libmhm_b200.so`` in-tree with nvcc for sm_100a.

The library is plain CUDA C++ with an ``extern "C"`` ABI (``include/mhm_b200.h``);
Python loads it with ctypes.  Usage: ``python -m pymhm_b200.build``.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SOURCES = ["q1_condense.cu", "skeleton.cu", "skeleton_static.cu", "batched_lu.cu", "p1_assembly.cu"]
LIBRARY = PKG / "libmhm_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libmhm_b200.so")
    return cand


def build(force: bool = False, verbose: bool = False) -> Path:
    srcs = [PKG / "csrc" / s for s in SOURCES]
    deps = srcs + [PKG / "csrc" / "mhm_common.cuh", ROOT / "include" / "mhm_b200.h"]
    if LIBRARY.exists() and not force:
        built = LIBRARY.stat().st_mtime
        if all(p.stat().st_mtime <= built for p in deps):
            return LIBRARY
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           f"-I{ROOT / 'include'}", "-diag-suppress", "177", "-o", str(tmp), *map(str, srcs)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + proc.stdout + proc.stderr)
    if verbose:
        sys.stderr.write(proc.stderr)
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
