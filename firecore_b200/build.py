"""Build recipe for the native library ``firecore_b200/libMMFFmulti_lib.so``.

Compiles every ``csrc/*.cu`` and ``csrc/*.cpp`` with nvcc for sm_100a and links
one shared library in-tree, so the built file travels with the source tree.
The C-ABI it exports is declared in ``include/MMFFmulti_lib.h``.

The seeded workload generator (``csrc/molgen.cpp``) is also linked on its own
into the host-only ``libmmff_gen.so`` (no CUDA): inputs for CPU-only consumers
(the reference timing arm) come from the same code without mapping the GPU
library.
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libMMFFmulti_lib.so")
GEN_LIB = os.path.join(HERE, "libmmff_gen.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
            "--expt-relaxed-constexpr", "-ccbin", HOST_CXX, "-I", os.path.join(ROOT, "include"),
            "-I", CSRC, "-Xptxas", "-warn-spills"]
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _needs(obj, srcs):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(s) > t for s in srcs)


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _needs(obj, [src] + headers):
            cmd = [NVCC] + ARCH + CU_FLAGS + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
        objs.append(obj)
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cpp"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _needs(obj, [src] + headers):
            cmd = [HOST_CXX] + CXX_FLAGS + ["-I", "/usr/local/cuda/include", "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
        objs.append(obj)
    if force or _needs(LIB, objs):
        # cudart is linked statically and loads the driver itself on first use,
        # so the library also loads (without computing) on hosts without a GPU.
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", HOST_CXX, "-Xcompiler", "-fopenmp", "-o", LIB] + objs + \
            ["-lcudart_static", "-lgomp"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    gen_src = os.path.join(CSRC, "molgen.cpp")
    if force or _needs(GEN_LIB, [gen_src] + headers):
        cmd = [HOST_CXX] + CXX_FLAGS + ["-shared", "-o", GEN_LIB, gen_src, "-lgomp"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
