"""Builds libd4core.so (sm_100a) and libd4umfpack.so in-tree.

Usage: python 2d4_b200/build.py [--jobs N]

Each .cu file under csrc/ compiles to an object with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; the FP64 files of
the plain form add ``--fmad=false`` so that no product-add is contracted into
an FMA (they keep the reference's rounding of every operation).  The objects
link into ``2d4_b200/lib/libd4core.so``.  ``umfpack/d4_umfpack.cpp`` (host
C++) links against it into ``2d4_b200/lib/libd4umfpack.so``, the
UMFPACK-compatible entry points, with an ``$ORIGIN`` run path.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
BUILD_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libd4core.so")
UMF_SRC = os.path.join(HERE, "umfpack", "d4_umfpack.cpp")
UMF_LIB = os.path.join(OUT_DIR, "libd4umfpack.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
# Files whose arithmetic must round like the reference's IEEE build.
NO_FMA = {"d4_fp64.cu", "d4_lu64.cu", "d4_lu_coop64.cu", "d4_ensemble.cu"}


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def compile_one(src):
    obj = os.path.join(BUILD_DIR, src[:-3] + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "d4core.h"))
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj
    flags = list(COMMON)
    if src in NO_FMA:
        flags.append("--fmad=false")
    cmd = [nvcc()] + ARCH + flags + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj


def build(jobs=8):
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(compile_one, sources()))
    if not (os.path.exists(LIB) and
            all(os.path.getmtime(LIB) >= os.path.getmtime(o) for o in objs)):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    build_umfpack()
    return LIB


def build_umfpack():
    deps = [UMF_SRC, LIB, os.path.join(ROOT, "include", "d4umfpack.h")]
    if os.path.exists(UMF_LIB) and all(os.path.getmtime(UMF_LIB) >= os.path.getmtime(d)
                                       for d in deps):
        return UMF_LIB
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I" + os.path.join(ROOT, "include"),
           "-o", UMF_LIB, UMF_SRC, "-L" + OUT_DIR, "-ld4core", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("g++ failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return UMF_LIB


if __name__ == "__main__":
    jobs = 8
    if "--jobs" in sys.argv:
        jobs = int(sys.argv[sys.argv.index("--jobs") + 1])
    print(build(jobs))
