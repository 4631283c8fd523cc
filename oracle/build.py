"""Build the CPU oracle library ``oracle/libqsim_oracle.so`` (test infrastructure).

``python oracle/build.py`` -- gcc, -O3, OpenMP, x86-64-v3 (AVX2/FMA) so the library
built here also runs on the GPU host.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libqsim_oracle.so")


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "cpu_kernels.c")
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(src):
        return LIB
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-o", LIB, src]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
