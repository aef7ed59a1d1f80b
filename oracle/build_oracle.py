"""Build recipe for the CPU oracle (test infrastructure).

Compiles oracle/qjx_oracle.c, oracle/fbasis_oracle.c and oracle/lpn_oracle.c into oracle/_build/liboracle.so.
The flags are part of the arithmetic contract shared with the CUDA engine:
-ffp-contract=off keeps every expression literal, so only explicit fma() calls fuse.
x86-64-v3 (AVX2 + FMA) keeps the library portable to the GPU box's host CPU.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
SOURCES = ["qjx_oracle.c", "fbasis_oracle.c", "lpn_oracle.c"]


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, s) for s in SOURCES if os.path.exists(os.path.join(HERE, s))]
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB):
        newest = max(os.path.getmtime(s) for s in srcs + [os.path.join(HERE, "qjx_oracle.h")])
        if os.path.getmtime(LIB) >= newest:
            return LIB
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-std=c11",
           "-shared", "-fPIC", "-o", LIB] + srcs + ["-lm"]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
