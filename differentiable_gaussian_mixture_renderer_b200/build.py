"""Builds libdgmr_b200.so (sm_100a) in-tree with nvcc.

    python -m differentiable_gaussian_mixture_renderer_b200.build

The kernels are compiled with -fmad=false and IEEE division / square root:
tile rectangles, depth keys and blended colours then follow one rounding
sequence that a CPU build can reproduce bit for bit.  Host code is compiled
with -ffp-contract=off for the same reason (the 4x4 inverse of the camera).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(OUT_DIR, "libdgmr_b200.so")
SOURCES = ["dgmr_splat.cu", "dgmr_marcher.cu", "dgmr_raster.cu", "dgmr_server.cpp", "dgmr_autotune.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDE = os.path.join(HERE, "..", "include")
VIEWER_SRC = os.path.join(HERE, "viewer", "headless_view.cpp")
VIEWER_PATH = os.path.join(OUT_DIR, "dgmr_headless_view")


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libdgmr_b200.so")


def host_compiler() -> list[str]:
    # the system g++ (the environment's CXX may point at a toolchain nvcc does not accept)
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def sources_newer_than(path: str) -> bool:
    if not os.path.exists(path):
        return True
    t = os.path.getmtime(path)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "dgmr_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not sources_newer_than(LIB_PATH):
        return LIB_PATH
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc(), *host_compiler(), "-std=c++17", "-O3", *ARCH, "-lineinfo", "-fmad=false", "-prec-div=true",
           "-prec-sqrt=true", "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared", "-o", tmp,
           *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


def build_viewer(force: bool = False) -> str:
    """The headless viewer (viewer/headless_view.cpp): host code over the C++
    viewer interface, linked against libdgmr_b200.so next to it."""
    lib = build(force=force)
    deps = [VIEWER_SRC, lib, os.path.join(INCLUDE, "dgmr_b200_sibr.hpp"), os.path.join(INCLUDE, "dgmr_b200.h")]
    if not force and os.path.exists(VIEWER_PATH) and all(os.path.getmtime(d) <= os.path.getmtime(VIEWER_PATH)
                                                          for d in deps):
        return VIEWER_PATH
    tmp = VIEWER_PATH + ".tmp"
    cmd = [nvcc(), *host_compiler(), "-Wno-deprecated-gpu-targets", "-std=c++17", "-O2", "-I", INCLUDE, VIEWER_SRC, "-L", OUT_DIR, "-ldgmr_b200",
           "-Xlinker", "-rpath,$ORIGIN", "-o", tmp]
    subprocess.run(cmd, check=True)
    os.replace(tmp, VIEWER_PATH)
    return VIEWER_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
    print(build_viewer(force="--force" in sys.argv))
