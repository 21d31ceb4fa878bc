"""Builds xenon_b200/lib/libxenon_b200.so (host C++ + sm_100a CUDA) in-tree.

Host scene code is compiled by g++ without FMA contraction (the BVH build must produce the
reference's node arrays bit for bit); the CUDA translation units are compiled for sm_100a only,
with -fmad=false on the path-tracing TU (the traversal and shading arithmetic keep the
reference's rounding) and FMA allowed in the guiding-network TU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
BUILDDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libxenon_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

CXX_SRCS = ["scene_host.cpp", "bvh_levels.cpp", "loaders.cpp", "capi_scene.cpp", "image_out.cpp"]
CU_STRICT = ["renderer.cu", "bvh_device.cu", "output_dev.cu"]
CU_FAST = ["guide.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _headers() -> list[str]:
    out = [os.path.join(INCLUDE, "xenon_b200.h")]
    for f in os.listdir(CSRC):
        if f.endswith((".h", ".cuh")):
            out.append(os.path.join(CSRC, f))
    return out


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILDDIR, exist_ok=True)
    nvcc = _nvcc()
    hdrs = _headers()
    objs = []
    for src in CXX_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILDDIR, src + ".o")
        if force or _stale(o, [s] + hdrs):
            _run([CXX, "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
                  "-Wextra", "-I", INCLUDE, "-c", s, "-o", o])
        objs.append(o)
    for src, strict in [(s, True) for s in CU_STRICT] + [(s, False) for s in CU_FAST]:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILDDIR, src + ".o")
        if force or _stale(o, [s] + hdrs):
            cmd = [nvcc, "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
                   "-I", INCLUDE, "-c", s, "-o", o]
            if strict:
                cmd[3:3] = ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
            if verbose_ptxas:
                cmd += ["-Xptxas", "-v"]
            _run(cmd)
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([nvcc, "-shared", *ARCH, "-o", LIB, *objs, "-lcudart_static", "-lpthread", "-ldl", "-lrt"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv)
