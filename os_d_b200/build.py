"""Build the native library os_d_b200/libqjx_b200.so (sm_100a) and the drop-in executable.

nvcc cross-compiles for sm_100a without a GPU.  The arithmetic contract of the engine
(bit-identical FP64 trajectories versus the CPU oracle) depends on two flags:
  -fmad=false        device code fuses only where __fma_rn is written
  -ffp-contract=off  host code fuses only where fma() is written
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libqjx_b200.so")
EXE = os.path.join(HERE, "qjx_b200")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
                  "-I", os.path.join(ROOT, "include")]
CXXFLAGS = ["-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-fPIC", "-std=c++17",
            "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include"]

CU_SOURCES = ["qjx_kernels.cu", "qjx_engine.cu", "fb_kernels.cu", "qjx_lpn.cu", "qjx_tree.cu"]
CXX_SOURCES = ["qjx_model.cpp", "qjx_config.cpp", "fb_model.cpp"]
EXE_SOURCES = ["qjx_main.cpp"]
HEADERS = ["qjx_device.cuh", "qjx_split.cuh", "qjx_config.h"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build(force=False, verbose=False, ptxas_info=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "qjx_b200.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        if not os.path.exists(s):
            continue
        o = os.path.join(OBJ, src + ".o")
        if force or _newer(o, [s] + headers):
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            _run([NVCC] + NVFLAGS + extra + ["-c", s, "-o", o], verbose)
        objs.append(o)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _newer(o, [s] + headers):
            _run(["g++"] + CXXFLAGS + ["-c", s, "-o", o], verbose)
        objs.append(o)
    if force or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fopenmp", "-cudart", "static"],
             verbose)
    exe_srcs = [os.path.join(CSRC, s) for s in EXE_SOURCES]
    if all(os.path.exists(s) for s in exe_srcs) and (force or _newer(EXE, exe_srcs + headers + [LIB])):
        _run(["g++"] + CXXFLAGS + exe_srcs + ["-o", EXE, "-L", HERE, "-lqjx_b200", "-Wl,-rpath,$ORIGIN",
                                              "-fopenmp"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
