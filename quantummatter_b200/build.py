"""Builds libqmb200.so in-tree with nvcc for sm_100a.

    python -m quantummatter_b200.build          # build if sources changed
    python -m quantummatter_b200.build --force  # rebuild

The library is plain CUDA C++ with a C ABI (include/qm_b200.h); nothing here goes
through torch's extension machinery.  The CUDA runtime is linked statically so the
shared object only needs the NVIDIA driver at load time.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libqmb200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libqmb200.so")


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _stale() -> bool:
    if not LIB.exists():
        return True
    built = LIB.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    deps.append(Path(__file__))
    return any(p.stat().st_mtime > built for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles every CUDA/C++ source of the library into quantummatter_b200/libqmb200.so."""
    if not force and not _stale():
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, *FLAGS, "-shared", "-I", str(INCLUDE), "-I", str(CSRC), "-o", str(tmp),
           *[str(s) for s in sources()], "-cudart", "static", "-lpthread", "-ldl"]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


def build_oracle() -> Path:
    """Builds the CPU oracle (test infrastructure) with its Makefile."""
    oracle = ROOT / "oracle"
    res = subprocess.run(["make", "-s", "-C", str(oracle)], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return oracle / "liboracle.so"


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force, verbose=True))
