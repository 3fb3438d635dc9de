"""Compile the sm_100a library ``libp2c_b200.so`` in place.

Every ``csrc/*.cu`` file is compiled with nvcc for ``sm_100a`` only
(``-gencode arch=compute_100a,code=sm_100a``) into ``_build/`` and linked into
``p2cccd_b200/libp2c_b200.so``, next to the Python host layer, so the shared
object travels with the source tree.  ``--fmad=false`` is a second guard next
to the explicitly rounded intrinsics in the certifier: no FMA contraction.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
ROOT = PKG_DIR.parent  # p2c-ccd_b200/
CSRC = ROOT / "csrc"
INCLUDE = ROOT.parent / "include"
BUILD = ROOT / "_build"
LIB = PKG_DIR / "libp2c_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the sm_100a library cannot be built")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> Path:
    """Build (incrementally) and return the path of libp2c_b200.so."""
    nvcc = _nvcc()
    BUILD.mkdir(parents=True, exist_ok=True)
    newest_header = max((p.stat().st_mtime for p in _headers()), default=0.0)
    objects = []
    for src in sorted(CSRC.glob("*.cu")):
        obj = BUILD / (src.stem + ".o")
        objects.append(obj)
        stale = force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header)
        if not stale:
            continue
        cmd = [nvcc, *NVCC_FLAGS, f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(src), "-o", str(obj)]
        if ptxas_info:
            cmd[1:1] = ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    link_stale = force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objects)
    if link_stale:
        cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(LIB),
               *map(str, objects), "-lcudart"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
