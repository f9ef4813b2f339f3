"""Build recipe of the native library (run by ``__graft_entry__.build()``).

Compiles the CUDA kernels and the C ABI for sm_100a with nvcc into
``multilayersolver2024_b200/libmlxpbd.so`` (in-tree, so the library travels with
the source tree), plus the headless mex gateway used by the boundary tests.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
MEX = PKG / "mex"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libmlxpbd.so"
MEXLIB = PKG / "mex" / "libmexLayerSolve3D.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
                     "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _stale(target: Path, sources) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(s).stat().st_mtime > t for s in sources)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build(verbose: bool = False, force: bool = False) -> Path:
    sources = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    deps = sources + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [INCLUDE / "mlxpbd.h"]
    if force or _stale(LIB, deps):
        tmp = LIB.with_suffix(".so.tmp")
        _run([_nvcc(), *NVCC_FLAGS, "-shared", "-o", tmp, *sources], verbose)
        os.replace(tmp, LIB)
    mex_src = [MEX / "mexLayerSolve3D.cpp", MEX / "mxshim.cpp"]
    if all(p.exists() for p in mex_src) and (force or _stale(MEXLIB, mex_src + [MEX / "mex.h", LIB])):
        tmp = MEXLIB.with_suffix(".so.tmp")
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wl,-Bsymbolic",
              f"-I{MEX}", f"-I{INCLUDE}", "-o", tmp, *mex_src,
              f"-L{PKG}", "-lmlxpbd", f"-Wl,-rpath,{PKG}"], verbose)
        os.replace(tmp, MEXLIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
