"""Build the sm_100a shared library ``cellgpu_b200/libcellgpu_b200.so`` in-tree with nvcc."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcellgpu_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(HERE, "..", "include", "cellgpu_b200.h")]
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-o", LIB, os.path.join(CSRC, "system.cu")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.check_call(cmd)
    return LIB


CPP = os.path.join(HERE, "cpp")
CPP_PROGRAMS = ["api_check", "voronoi_example"]
CUDA_INCLUDE = os.environ.get("CUDA_INCLUDE", "/usr/local/cuda/include")


def build_cpp(force: bool = False) -> list:
    """The C++ class-API programs (cellgpu_b200/cpp), linked against the in-tree library."""
    out = []
    inc = os.path.join(HERE, "..", "include")
    for name in CPP_PROGRAMS:
        src = os.path.join(CPP, name + ".cpp")
        exe = os.path.join(CPP, name)
        deps = [src, os.path.join(CPP, "cellgpu.hpp"), LIB]
        if force or not os.path.exists(exe) or any(os.path.getmtime(d) > os.path.getmtime(exe) for d in deps):
            subprocess.check_call([os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-Wall", "-I", inc,
                                   "-I", CUDA_INCLUDE, src, "-o", exe, "-L", HERE, "-lcellgpu_b200",
                                   "-Wl,-rpath,$ORIGIN/.."])
        out.append(exe)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    build_cpp(force="--force" in sys.argv)
    print(LIB)
