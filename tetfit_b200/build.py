"""Build recipe for libtetfit_b200.so (sm_100a, in-tree) and the `tetfit`
command-line driver linked against it.

    python -m tetfit_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libtetfit_b200.so")
CLI = os.path.join(HERE, "tetfit")
CLI_SOURCE = os.path.join(CSRC, "tetfit_main.cpp")
SOURCES = ["script.cpp", "fit.cpp", "fit_kernels.cu", "tet.cpp", "tet_kernels.cu", "tet_group.cpp",
           "tet_group_kernels.cu", "mlp.cu", "pcg.cu", "dt_gpu.cu", "barrier_check.cu", "capi.cpp", "capi_batch.cpp"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]
OBJ_DIR = os.path.join(HERE, "_build")


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "tetfit.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_cli(verbose: bool = False) -> str:
    """`tetfit` driver: links libtetfit_b200.so from its own folder."""
    cxx = os.environ.get("CXX", "g++")
    cmd = [cxx, "-O2", "-std=c++17", CLI_SOURCE, "-o", CLI + ".tmp", "-L" + HERE, "-l:libtetfit_b200.so",
           "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=HERE)
    os.replace(CLI + ".tmp", CLI)
    return CLI


def build(force: bool = False, verbose: bool = False) -> str:
    if force or needs_build():
        nvcc = os.environ.get("NVCC", "nvcc")
        os.makedirs(OBJ_DIR, exist_ok=True)
        objs = [os.path.join(OBJ_DIR, os.path.splitext(s)[0] + ".o") for s in SOURCES]

        def compile_one(src_obj):
            cmd = [nvcc] + NVCC_FLAGS + ["-c", src_obj[0], "-o", src_obj[1]]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True, cwd=CSRC)

        # one nvcc per source file, in parallel, then one link
        with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
            list(ex.map(compile_one, zip(sources(), objs)))
        cmd = [nvcc] + NVCC_FLAGS + ["-shared"] + objs + ["-o", OUT + ".tmp"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=CSRC)
        os.replace(OUT + ".tmp", OUT)
    if force or not os.path.exists(CLI) or os.path.getmtime(CLI) < max(os.path.getmtime(OUT),
                                                                        os.path.getmtime(CLI_SOURCE)):
        build_cli(verbose)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
