"""Build recipe for the CPU oracle (test infrastructure only).

Produces oracle/_build/libtf_oracle.so (strict IEEE FP64, the parity checker)
and oracle/_build/libtf_oracle_omp.so (same source with OpenMP loops, timed as
the CPU baseline).  The reference itself cannot be compiled here (it needs
Eigen3, Spectra, GSL, Silo and Boost, none of which is installed), so there is
no oracle/_ref build.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
SOURCES = ["script.cpp", "fit.cpp", "tet.cpp", "capi.cpp"]
LIB = os.path.join(OUT_DIR, "libtf_oracle.so")
LIB_OMP = os.path.join(OUT_DIR, "libtf_oracle_omp.so")


def _stale(out):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(os.path.join(HERE, f)) > t
               for f in os.listdir(HERE) if f.endswith((".cpp", ".hpp")))


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    base = ["g++", "-std=c++17", "-fPIC", "-shared", "-Wall", "-Wno-unused-function", "-Wno-unknown-pragmas"]
    if force or _stale(LIB):
        subprocess.run(base + ["-O2"] + srcs + ["-o", LIB + ".tmp"], check=True)
        os.replace(LIB + ".tmp", LIB)
    if force or _stale(LIB_OMP):
        subprocess.run(base + ["-O3", "-fopenmp"] + srcs + ["-o", LIB_OMP + ".tmp"], check=True)
        os.replace(LIB_OMP + ".tmp", LIB_OMP)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
