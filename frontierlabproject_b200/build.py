"""Build ``libqsim_b200.so`` in-tree with nvcc for sm_100a.

    python -m frontierlabproject_b200.build [--force] [--verbose]

Objects go to ``frontierlabproject_b200/_build/``; the shared library is written next to
this file so it travels with the source tree.  The library links the CUDA runtime
statically and exports only the C ABI of ``include/qsim_b200.h``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libqsim_b200.so")
SOURCES = ["kern_pass.cu", "kern_gate.cu", "kern_adjoint.cu", "kern_batch.cu", "kern_dense_tc.cu", "kern_sample.cu",
           "state.cu", "plan.cpp", "jit.cpp", "batch.cpp", "lqr.cpp", "fuse.cpp", "prep.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps_mtime() -> float:
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(REPO, "include", "qsim_b200.h"))
    return max(os.path.getmtime(f) for f in files if os.path.exists(f))


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _deps_mtime():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    common = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "-I", os.path.join(REPO, "include"), "--expt-relaxed-constexpr"] + ARCH
    if verbose:
        common += ["-Xptxas", "-v"]
    common += list(extra_flags or [])

    def compile_one(src):
        obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        cmd = [cc, "-c", os.path.join(CSRC, src), "-o", obj] + common
        if src.endswith(".cpp"):
            cmd = [cc, "-x", "cu", "-c", os.path.join(CSRC, src), "-o", obj] + common
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        return obj, r.stderr

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    if verbose:
        for _, log in results:
            sys.stderr.write(log)
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    cmd = [cc, "-shared", "-o", tmp] + objs + ARCH + ["-Xcompiler", "-fPIC", "-cudart", "static", "-ldl",
                                                        "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
