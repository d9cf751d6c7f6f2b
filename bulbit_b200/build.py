"""Builds libbulbit_b200.so in-tree: CUDA sources for sm_100a with nvcc, host
C++ with g++, linked into one shared library next to this file.

Kernels are compiled with --fmad=false (no FMA contraction) and IEEE division
and square root, which the bit-exact parity with the reference's x86-64 float
arithmetic relies on.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbulbit_b200.so")
INCLUDE = os.path.join(ROOT, "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
                     "-std=c++20", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC]
CXX_FLAGS = ["-O2", "-std=c++20", "-fPIC", "-pthread", "-I" + INCLUDE, "-I" + CSRC,
             "-I" + os.path.join(CUDA_HOME, "include")]

CU_SOURCES = ["accel.cu", "render.cu", "noalloc.cu", "guide.cu", "lbvh.cu", "sah_build.cu", "split_build.cu"]
CXX_SOURCES = ["host_build.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "bbg.h"))
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC] + NVCC_FLAGS + extra + ["-c", s, "-o", o])
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            jobs.append(["g++"] + CXX_FLAGS + ["-c", s, "-o", o])
    out = []
    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        for text in ex.map(_run, jobs):
            out.append(text)
    if jobs or not os.path.exists(LIB):
        tmp = LIB + ".tmp"
        _run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lpthread"])
        shutil.move(tmp, LIB)
    if verbose:
        print("\n".join(o for o in out if o.strip()))
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
    print(LIB)
