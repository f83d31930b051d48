"""Builds the evaluator library libgrn_b200.so in-tree.

  python grn-gpu-performance_b200/build.py [--force] [--verbose]

CUDA sources are compiled for sm_100a only
(nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo), host sources with
g++; everything links into lib/libgrn_b200.so with the CUDA runtime linked
statically, so the library loads without a CUDA toolkit on the library path.
The ptxas resource report (registers, spills, shared memory per kernel) is
written to _build/ptxas.log.  lib/libgrn_b200_checked.so is the same library
with the simulation kernel built with GRN_BOUNDS_CHECK=1 (every state access
checked; for the tests).
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libgrn_b200.so")
# The same library with every state access of the simulation kernel
# bounds-checked (GRN_BOUNDS_CHECK, tests only).
CHECKED_LIB = os.path.join(LIB_DIR, "libgrn_b200_checked.so")
KERNEL_SRC = os.path.join(HERE, "csrc", "grn_sim_kernel.cu")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
CPP_SOURCES = sorted(glob.glob(os.path.join(HERE, "host", "*.cpp")))
HEADERS = (sorted(glob.glob(os.path.join(HERE, "csrc", "*.h")))
           + sorted(glob.glob(os.path.join(HERE, "host", "*.h")))
           + [os.path.join(ROOT, "include", "grn_gpu.h")])


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose, log=None):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if log is not None:
        log.append(r.stdout)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r.stdout


def build(force=False, verbose=False):
    if not os.path.exists(NVCC) and shutil.which("nvcc") is None:
        raise RuntimeError("nvcc not found; set CUDA_HOME")
    nvcc = NVCC if os.path.exists(NVCC) else shutil.which("nvcc")
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    objs = []
    ptxas_log = []
    for src in CU_SOURCES:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _newer(obj, [src] + HEADERS):
            _run([nvcc] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                                  "-Xptxas", "-v", "--expt-relaxed-constexpr",
                                  "-c", src, "-o", obj], verbose, ptxas_log)
    for src in CPP_SOURCES:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _newer(obj, [src] + HEADERS):
            _run(["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-pthread",
                  "-I" + os.path.join(CUDA_HOME, "include"), "-c", src, "-o", obj], verbose)
    if ptxas_log:
        with open(os.path.join(BUILD, "ptxas.log"), "w") as f:
            f.write("\n".join(ptxas_log))
    if force or _newer(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs
             + ["-cudart", "static", "-Xcompiler", "-pthread", "-lrt", "-ldl"], verbose)
    checked_obj = os.path.join(BUILD, "grn_sim_kernel_checked.cu.o")
    if force or _newer(checked_obj, [KERNEL_SRC] + HEADERS):
        _run([nvcc] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                              "--expt-relaxed-constexpr", "-DGRN_BOUNDS_CHECK=1",
                              "-c", KERNEL_SRC, "-o", checked_obj], verbose)
    checked_objs = [checked_obj if o.endswith("grn_sim_kernel.cu.o") else o for o in objs]
    if force or _newer(CHECKED_LIB, checked_objs):
        _run([nvcc] + ARCH + ["-shared", "-o", CHECKED_LIB] + checked_objs
             + ["-cudart", "static", "-Xcompiler", "-pthread", "-lrt", "-ldl"], verbose)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
