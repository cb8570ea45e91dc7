"""Build recipe for the oracle shared library (test infrastructure only).

Compiles ferray_cpu.c (restatement of ferray's CPU GEMM) and dd_oracle.c
(double-double reference) into oracle/liboracle.so with gcc.

-ffp-contract=off keeps every `a*b + c` that the restated Rust code writes as
two roundings from being fused by the C compiler; the explicit fma() calls
(Rust `mul_add` and the AVX2 `vfmadd` lanes) stay fused.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SOURCES = [os.path.join(HERE, "ferray_cpu.c"), os.path.join(HERE, "dd_oracle.c")]


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB):
        newest = max(os.path.getmtime(s) for s in SOURCES + [__file__])
        if os.path.getmtime(LIB) >= newest:
            return LIB
    cmd = ["gcc", "-O3", "-mavx2", "-mfma", "-ffp-contract=off", "-fopenmp",
           "-fPIC", "-shared", "-o", LIB] + SOURCES + ["-lm"]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
