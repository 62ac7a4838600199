"""Builds libhenon_b200.so (CUDA kernels + C ABI) and the pybind11 module
henon_map_engine in-tree, for sm_100a only.

Usage: python -m henon_map_cpp_b200.build [--force]

Objects go to <repo>/_build/; the shared libraries are written next to this
file so that they travel with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
BUILD = REPO / "_build"
INCLUDE = REPO / "include"
LIB = PKG / "libhenon_b200.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: no implicit contraction of a*b+c anywhere in device code.
# The kernels spell their arithmetic explicitly (__d*_rn for the exact
# path, fma() for the fast one); the flag makes CUDA's own libm (log, log10,
# atan2) compile exactly as in the reference's --fmad=false build.
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--fmad=false",
              "-Xptxas", "-O3", *ARCH, f"-I{INCLUDE}"]
# Host code: no -march and no contraction, so host doubles are plain SSE2
# binary64 arithmetic like the reference's host build.
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
             f"-I{CUDA_HOME / 'include'}", f"-I{INCLUDE}"]

CU_SOURCES = ["track.cu", "noalloc.cu", "tangent.cu", "fused.cu", "ghosts.cu", "batch.cu",
              "adjoint.cu", "tunes.cu"]
CPP_SOURCES = ["capi.cpp", "modulation.cpp", "indicators.cpp", "particles_extra.cpp",
               "batch.cpp", "adjoint.cpp", "tunes.cpp", "fft_plan.cpp"]


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def build_library(force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    objs = []
    hdrs = _headers()
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".cu.o")
        if force or _stale(o, [s, *hdrs]):
            _run([NVCC, *NVCC_FLAGS, "-c", str(s), "-o", str(o)])
        objs.append(o)
    for src in CPP_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".cpp.o")
        if force or _stale(o, [s, *hdrs]):
            _run(["g++", *CXX_FLAGS, "-c", str(s), "-o", str(o)])
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([NVCC, "-shared", *ARCH, "-o", str(LIB), *map(str, objs),
              "-lcudart", "-lcufft", "-lpthread"])
    return LIB


def build_engine(force: bool = False) -> Path | None:
    """pybind11 module `henon_map_engine` over the C ABI."""
    src = CSRC / "bind.cpp"
    if not src.exists():
        return None
    import pybind11  # noqa: PLC0415

    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    out = PKG / f"henon_map_engine{suffix}"
    if force or _stale(out, [src, LIB, *_headers()]):
        py_inc = sysconfig.get_paths()["include"]
        _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
              f"-I{pybind11.get_include()}", f"-I{py_inc}", f"-I{INCLUDE}",
              f"-I{CUDA_HOME / 'include'}", str(src), "-o", str(out),
              f"-L{PKG}", "-lhenon_b200", "-Wl,-rpath,$ORIGIN"])
    return out


def build_all(force: bool = False) -> None:
    build_library(force)
    build_engine(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
