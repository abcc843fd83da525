"""Build recipe of the oracle's C++ CPU arm (TEST INFRASTRUCTURE).

``python -m oracle.build_cpu_ref`` compiles ``oracle/cpu_ref.cpp`` with
g++ -O3, OpenMP and numpy's bundled OpenBLAS (scipy_openblas64) into
``oracle/_build/libcpu_ref.so``.  x86-64-v3 (AVX2 + FMA) rather than
-march=native, so a library built on one host runs on another; the BLAS
kernels pick their own instruction set at run time.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_ref.cpp")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libcpu_ref.so")


def openblas_path():
    import numpy
    libs = glob.glob(os.path.join(os.path.dirname(numpy.__file__), os.pardir, "numpy.libs",
                                  "libscipy_openblas64_*.so*"))
    if not libs:
        raise RuntimeError("numpy's bundled scipy_openblas64 library was not found")
    return os.path.realpath(libs[0])


def build(force=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    blas = openblas_path()
    cmd = ["g++", "-O3", "-march=x86-64-v3", "-fopenmp", "-shared", "-fPIC", "-std=c++17", "-o", LIB + ".tmp",
           SRC, blas, f"-Wl,-rpath,{os.path.dirname(blas)}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed ({r.returncode}):\n{r.stderr[-4000:]}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
