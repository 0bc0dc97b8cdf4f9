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
SOURCES = ["q1_condense.cu", "skeleton.cu", "skeleton_static.cu", "batched_lu.cu", "p1_assembly.cu",
           "general_pcg.cu", "dense_local.cu", "p2_local.cu"]
LIBRARY = PKG / "libmhm_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libmhm_b200.so")
    return cand


def _compile(src: Path, obj: Path, verbose: bool) -> str:
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", f"-I{ROOT / 'include'}",
           "-diag-suppress", "177", "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n" + proc.stdout + proc.stderr)
    return proc.stderr


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every source to an object in ``_build/`` (in parallel, only the ones whose
    source or headers changed) and link ``libmhm_b200.so``."""
    from concurrent.futures import ThreadPoolExecutor

    srcs = [PKG / "csrc" / s for s in SOURCES]
    headers = [PKG / "csrc" / "mhm_common.cuh", ROOT / "include" / "mhm_b200.h"]
    objdir = ROOT / "_build"
    objdir.mkdir(exist_ok=True)
    objs = [objdir / (p.stem + ".o") for p in srcs]
    newest_header = max(h.stat().st_mtime for h in headers)
    stale = [(s, o) for s, o in zip(srcs, objs)
             if force or not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, newest_header)]
    if not stale and LIBRARY.exists() and all(o.stat().st_mtime <= LIBRARY.stat().st_mtime for o in objs):
        return LIBRARY
    with ThreadPoolExecutor(max_workers=max(1, min(len(stale), os.cpu_count() or 1))) as pool:
        logs = list(pool.map(lambda so: _compile(so[0], so[1], verbose), stale))
    if verbose:
        for log in logs:
            sys.stderr.write(log)
    tmp = LIBRARY.with_suffix(".so.tmp")
    proc = subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs)], capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + proc.stdout + proc.stderr)
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
