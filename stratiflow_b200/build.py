"""Build recipe of the CUDA library ``libstratiflow_b200.so`` (sm_100a only).

    python -m stratiflow_b200.build [--verbose]

compiles ``csrc/*.cu`` with nvcc into the package directory, so the library
travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libstratiflow_b200.so")
SOURCES = ["sf_solver.cu", "sf_kernels.cu", "sf_noalloc.cu", "sf_vecs.cu", "sf_net.cu", "sf_io.cu", "sf_adjoint.cu", "sf_xmarch.cu", "sf_zstep.cu", "sf_zstep2.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _inputs():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h"))]
    files.append(os.path.join(HERE, "..", "include", "stratiflow_b200.h"))
    return files


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _inputs())


HOST = os.path.join(HERE, "host")
HOST_LIB = os.path.join(HERE, "libstratiflow_host.so")


def build_host(force: bool = False) -> str:
    """The C++ drivers (host/stratiflow.hpp, host/sf_host.cpp), linked against
    libstratiflow_b200.so."""
    srcs = [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith((".cpp", ".hpp"))]
    if (not force and os.path.exists(HOST_LIB)
            and all(os.path.getmtime(f) <= os.path.getmtime(HOST_LIB) for f in srcs + [LIB])):
        return HOST_LIB
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", os.path.join(HERE, "..", "include"),
           os.path.join(HOST, "sf_host.cpp"), "-L", HERE, "-lstratiflow_b200", "-Wl,-rpath,$ORIGIN",
           "-o", HOST_LIB]
    subprocess.check_call(cmd)
    return HOST_LIB


OBJ = os.path.join(HERE, "..", "_build", "obj")


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src).replace(".cu", ".o"))
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-c", "-Xcompiler", "-fPIC",
           "--expt-relaxed-constexpr", "-o", obj, src]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    subprocess.check_call(cmd)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every translation unit (in parallel; one object per source
    under _build/) and link them into the package's shared library."""
    if force or needs_build():
        from concurrent.futures import ThreadPoolExecutor
        os.makedirs(OBJ, exist_ok=True)
        srcs = [os.path.join(CSRC, s) for s in SOURCES]
        with ThreadPoolExecutor(max_workers=len(srcs)) as ex:
            objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
        subprocess.check_call([NVCC, *ARCH, "-shared", "-o", LIB, *objs])
    build_host(force)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="--verbose" in sys.argv)
    print(LIB)
