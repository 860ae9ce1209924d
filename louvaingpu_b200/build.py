"""Build recipe for liblvg.so (sm_100a) and the host graph generators.

    python -m louvaingpu_b200.build            # build what is out of date
    python -m louvaingpu_b200.build --force    # rebuild everything

The CUDA library is compiled with nvcc for sm_100a only and written in-tree
(louvaingpu_b200/liblvg.so) so that it travels with the source tree.
"""
import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "liblvg.so")
GENLIB = os.path.join(HERE, "liblvggen.so")

CU_SOURCES = ["prims.cu", "louvain.cu", "induce.cu", "capi.cu", "noalloc.cu", "gen_device.cu", "server.cu"]
CU_HEADERS = ["lvg_internal.cuh", "prims.cuh", "louvain.cuh"]
GEN_SOURCES = ["gen_host.cpp"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
    "-fmad=false",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lvg(force=False, verbose=False):
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in CU_HEADERS] + [os.path.join(INCLUDE, "lvg.h"), __file__]
    if not force and not _stale(LIB, deps):
        return LIB
    nvcc = _nvcc()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = [nvcc, *NVCC_FLAGS, "-I", INCLUDE, "-c", s, "-o", o]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        objs.append(o)
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs,
                           "-o", tmp, "-lcudart"])
    os.replace(tmp, LIB)
    return LIB


def build_gen(force=False):
    srcs = [os.path.join(CSRC, s) for s in GEN_SOURCES]
    deps = srcs + [os.path.join(CSRC, "gen_host.h"), __file__]
    if not force and not _stale(GENLIB, deps):
        return GENLIB
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    tmp = GENLIB + ".tmp"
    subprocess.check_call([cxx, "-O3", "-march=x86-64-v3", "-std=c++17", "-fPIC", "-shared", "-fopenmp",
                           "-I", INCLUDE, *srcs, "-o", tmp])
    os.replace(tmp, GENLIB)
    return GENLIB


def build_all(force=False, verbose=False):
    build_gen(force)
    return build_lvg(force, verbose)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build_all(a.force, a.verbose))
    sys.exit(0)
