"""Builds the in-tree shared library ``lsim_b200/libfsimb200.so`` for sm_100a.

C++ host sources are compiled with the system g++, CUDA sources with nvcc
(``-gencode arch=compute_100a,code=sm_100a -lineinfo``), and everything is
linked with nvcc against the static CUDA runtime.  Objects go to
``lsim_b200/_build/``.  Usage: ``python -m lsim_b200.build [--force]``.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfsimb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

CXX_SOURCES = ["fsimb_netlist.cpp", "fsimb_gen.cpp", "fsimb_plan.cpp"]
CU_SOURCES = ["fsimb_kernels.cu", "fsimb_engine.cu", "fsimb_batch.cu", "fsimb_serve.cu", "fsimb_loader.cu"]
HEADERS = ["fsimb_netlist.h", "fsimb_gen.h", "fsimb_plan.h", "fsimb_kernels.cuh", "fsimb_internal.h", "fsimb_batch.h",
           "fsimb_loader.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
APPS = ["fsimb_simple", "fsimb_ma_partition"]  # drop-ins for main/simple and MA_cuda_partition
BIN = os.path.join(HERE, "bin")


def _nvcc():
    for c in [os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")]:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build lsim_b200")


def _cxx():
    for c in ["/usr/bin/g++", shutil.which("g++")]:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("g++ not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compiles what changed; returns the library path."""
    os.makedirs(BUILD, exist_ok=True)
    nvcc, cxx = _nvcc(), _cxx()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "fsimb.h")]
    objs = []
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + hdrs):
            cmd = [cxx, "-std=c++17", "-O3", "-fPIC", "-Wall", "-I" + INCLUDE, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
        objs.append(o)
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + hdrs):
            cmd = [nvcc] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                                   "-ccbin", cxx, "-I" + INCLUDE, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
        objs.append(o)
    if force or _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-ccbin", cxx, "-cudart", "static", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    os.makedirs(BIN, exist_ok=True)
    for app in APPS:
        s = os.path.join(CSRC, "apps", app + ".cpp")
        exe = os.path.join(BIN, app)
        if force or _stale(exe, [s, LIB, os.path.join(INCLUDE, "fsimb.h")]):
            cmd = [cxx, "-std=c++17", "-O2", "-I" + INCLUDE, s, "-o", exe, "-L" + HERE,
                   "-lfsimb200", "-Wl,-rpath,$ORIGIN/.."]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
