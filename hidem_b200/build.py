"""Build recipe of libhidem_b200.so (in-tree, sm_100a).

    python -m hidem_b200.build          # rebuilds when a source is newer than the library

The CUDA sources are compiled with ``-fmad=false`` and IEEE division / square root
(no ``--use_fast_math``): the per-pair, per-side and integrate arithmetic must round
exactly like the reference's IEEE build for the bit-exact parity tests.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libhidem_b200.so"
OBJ = PKG / "_build"

CU_SOURCES = ["kernels.cu", "api.cu", "noalloc.cu", "surrogate.cu", "mesh.cu"]
CPP_SOURCES = ["lattice.cpp", "config.cpp", "h5lite.cpp", "checkpoint.cpp", "particle_file.cpp"]
HEADERS = ["internal.h", "kernels.h", "physics.cuh", "h5lite.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-prec-div=true",
              "-prec-sqrt=true", "-ftz=false", "-Xcompiler", "-fPIC,-O3"]


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(cuda) / "bin" / "nvcc"
    return str(cand) if cand.exists() else (shutil.which("nvcc") or "nvcc")


def _gxx() -> str:
    # the system compiler: CC/CXX in some environments point at wrappers without OpenMP
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else (shutil.which("g++") or "g++")


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in CU_SOURCES + CPP_SOURCES + HEADERS] + [INCLUDE / "hidem_b200.h"]
    return any(p.stat().st_mtime > t for p in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} (exit {r.returncode})")


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every CUDA / C++ source of the package into ``libhidem_b200.so``."""
    if not force and not _stale():
        return LIB
    OBJ.mkdir(exist_ok=True)
    nvcc, gxx = _nvcc(), _gxx()
    objs = []
    for src in CU_SOURCES:
        obj = OBJ / (src + ".o")
        _run([nvcc, *ARCH, *NVCC_FLAGS, f"-I{INCLUDE}", "-c", str(CSRC / src), "-o", str(obj)])
        objs.append(str(obj))
    for src in CPP_SOURCES:
        obj = OBJ / (src + ".o")
        _run([gxx, "-std=c++17", "-O3", "-fPIC", "-fopenmp", f"-I{INCLUDE}", "-c",
              str(CSRC / src), "-o", str(obj)])
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc, *ARCH, "-shared", "-o", str(tmp), *objs, "-Xcompiler", "-fopenmp",
          f"-ccbin={gxx}", "-lz"])
    os.replace(tmp, LIB)
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
