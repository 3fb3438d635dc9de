"""Compile the sm_100a library ``libp2c_b200.so`` in place.

Every ``csrc/*.cu`` file is compiled with nvcc for ``sm_100a`` only
(``-gencode arch=compute_100a,code=sm_100a``) into ``_build/`` and linked into
``p2cccd_b200/libp2c_b200.so``, next to the Python host layer, so the shared
object travels with the source tree.  ``--fmad=false`` is a second guard next
to the explicitly rounded intrinsics in the certifier: no FMA contraction.

Staleness is decided by content, not by file times: every object records the
SHA-256 of its compile command, its source and every header, and the library
records the digest of all of them (``libp2c_b200.so.sha256``).  A tree copied
to another machine with prebuilt objects therefore rebuilds exactly what its
sources no longer match, and never links an object built from other sources.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
ROOT = PKG_DIR.parent  # p2c-ccd_b200/
CSRC = ROOT / "csrc"
INCLUDE = ROOT.parent / "include"
BUILD = ROOT / "_build"
LIB = PKG_DIR / "libp2c_b200.so"
LIB_DIGEST = LIB.with_name(LIB.name + ".sha256")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-Xcompiler", "-ffp-contract=off",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the sm_100a library cannot be built")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _digest(parts: list[bytes]) -> str:
    h = hashlib.sha256()
    for p in parts:
        h.update(len(p).to_bytes(8, "little"))
        h.update(p)
    return h.hexdigest()


def _read(path: Path) -> str | None:
    try:
        return path.read_text().strip()
    except OSError:
        return None


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False, jobs: int | None = None,
          extra_flags: list[str] | None = None, lib: Path | None = None, build_dir: Path | None = None) -> Path:
    """Build (incrementally) and return the path of the library.

    ``extra_flags``, ``lib`` and ``build_dir`` produce a variant library
    elsewhere (for example a measurement build with a macro set); the default
    is the product library."""
    nvcc = _nvcc()
    lib = LIB if lib is None else Path(lib)
    build_dir = BUILD if build_dir is None else Path(build_dir)
    lib_digest = lib.with_name(lib.name + ".sha256")
    build_dir.mkdir(parents=True, exist_ok=True)
    flags = NVCC_FLAGS + list(extra_flags or [])
    header_blob = [p.name.encode() + b"\0" + p.read_bytes() for p in _headers()]
    sources = sorted(CSRC.glob("*.cu"))
    jobs_list = []
    for src in sources:
        obj = build_dir / (src.stem + ".o")
        cmd = [nvcc, *flags, f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(src), "-o", str(obj)]
        if ptxas_info:
            cmd[1:1] = ["-Xptxas", "-v"]
        key = _digest([" ".join(flags).encode(), src.read_bytes(), *header_blob])
        jobs_list.append((src, obj, cmd, key))
    total = _digest([k.encode() for *_, k in jobs_list])
    if not force and lib.exists() and _read(lib_digest) == total:
        return lib

    def compile_one(job) -> None:
        src, obj, cmd, key = job
        stamp = obj.with_suffix(".sha256")
        if not force and obj.exists() and _read(stamp) == key:
            return
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        stamp.unlink(missing_ok=True)
        subprocess.run(cmd, check=True)
        stamp.write_text(key + "\n")

    n = jobs or min(len(jobs_list), max(1, os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=n) as pool:
        list(pool.map(compile_one, jobs_list))
    lib_digest.unlink(missing_ok=True)
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(lib),
           *(str(o) for _, o, _, _ in jobs_list), "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    lib_digest.write_text(total + "\n")
    return lib


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
