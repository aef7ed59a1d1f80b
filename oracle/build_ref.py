"""Build recipe for oracle/_ref/libfbref.so: the reference's own f-basis Lindblad solver.

Compiles the unmodified sources of source/cpp/CQdiss_os_dimer (CQdiss, SparceM_op, read_config)
where they lie in the reference tree, against oracle/ref_shim/mkl.h (the four MKL routines they
call, written from Intel's documented CSR semantics in oracle/ref_shim/mkl_shim.cpp), plus the
driver oracle/fbasis_ref_driver.cpp.  Output only into oracle/_ref/ (git-ignored).  Test
infrastructure: pins the f-basis oracle and the library's Liouvillian builder; nothing in the
product links it.  Skipped (returns None) when the reference tree is absent.
"""
import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libfbref.so")
REF = "/root/reference/source/cpp/CQdiss_os_dimer"
SUBDIRS = ["CQdiss", "SparceM_op", "read_config"]


def build(force: bool = False):
    if not os.path.isdir(REF):
        return None
    srcs = []
    for d in SUBDIRS:
        srcs += sorted(glob.glob(os.path.join(REF, d, "*.cpp")))
    mine = [os.path.join(HERE, "ref_shim", "mkl_shim.cpp"), os.path.join(HERE, "fbasis_ref_driver.cpp")]
    os.makedirs(OUT_DIR, exist_ok=True)
    deps = srcs + mine + [os.path.join(HERE, "ref_shim", "mkl.h")]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(s) for s in deps):
        return LIB
    inc = ["-I", os.path.join(HERE, "ref_shim")] + sum([["-I", os.path.join(REF, d)] for d in SUBDIRS], [])
    objs = []
    for s in srcs + mine:
        o = os.path.join(OUT_DIR, os.path.basename(os.path.dirname(s)) + "_" + os.path.basename(s) + ".o")
        std = "-std=c++17" if s in mine else "-std=c++11"  # the reference's Makefile builds it as C++11
        subprocess.check_call(["g++", std, "-O2", "-fPIC", "-fopenmp", "-w"] + inc + ["-c", s, "-o", o])
        objs.append(o)
    subprocess.check_call(["g++", "-shared", "-fopenmp", "-o", LIB] + objs)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
