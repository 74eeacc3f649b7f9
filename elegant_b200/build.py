"""Builds libtrkgpu.so in-tree (elegant_b200/libtrkgpu.so) for sm_100a.

The kernels translation unit is compiled twice: once without FMA contraction
(-fmad=false, the parity build that reproduces the reference's rounding) and
once with it (the fast build).  Host code is compiled without FMA contraction
so the per-element constants round like the reference's CPU code.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtrkgpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
INC = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

HEADERS = [os.path.join(ROOT, "include", "trk.h")] + [
    os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))
]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def objects():
    """(source, object, command) triples."""
    nv_common = [NVCC, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
                 "-Xptxas", "-v" if os.environ.get("TRK_PTXAS_VERBOSE") else "-O3"] + ARCH + INC
    out = []
    src = os.path.join(CSRC, "trk_kernels.cu")
    o = os.path.join(BUILD, "trk_kernels_exact.o")
    out.append((src, o, nv_common + ["-DTRK_FAST=0", "-fmad=false", "-c", src, "-o", o]))
    o = os.path.join(BUILD, "trk_kernels_fast.o")
    out.append((src, o, nv_common + ["-DTRK_FAST=1", "-fmad=true", "-c", src, "-o", o]))
    src = os.path.join(CSRC, "trk_api.cu")
    o = os.path.join(BUILD, "trk_api.o")
    out.append((src, o, nv_common + ["-c", src, "-o", o]))
    src = os.path.join(CSRC, "trk_compile.cpp")
    o = os.path.join(BUILD, "trk_compile.o")
    out.append((src, o, ["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math"] + INC +
                ["-c", src, "-o", o]))
    src = os.path.join(CSRC, "trk_aperture.cpp")
    o = os.path.join(BUILD, "trk_aperture.o")
    out.append((src, o, ["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math"] + INC +
                ["-c", src, "-o", o]))
    src = os.path.join(CSRC, "trk_comm.cpp")
    o = os.path.join(BUILD, "trk_comm.o")
    out.append((src, o, ["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off"] + INC +
                ["-I/usr/local/cuda/include", "-c", src, "-o", o]))
    src = os.path.join(CSRC, "trk_lattice.c")
    o = os.path.join(BUILD, "trk_lattice.o")
    out.append((src, o, ["gcc", "-std=gnu11", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math"] + INC +
                ["-c", src, "-o", o]))
    src = os.path.join(CSRC, "trk_observe.cu")
    o = os.path.join(BUILD, "trk_observe.o")
    out.append((src, o, nv_common + ["-fmad=false", "-c", src, "-o", o]))
    src = os.path.join(CSRC, "trk_noalloc.cu")
    o = os.path.join(BUILD, "trk_noalloc.o")
    out.append((src, o, nv_common + ["-c", src, "-o", o]))
    return out


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    objs, todo = [], []
    for src, o, cmd in objects():
        if _newer(o, [src] + HEADERS):
            todo.append(cmd)
        objs.append(o)
    # the translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(_run, cmd, verbose) for cmd in todo]:
            f.result()
    if _newer(LIB, objs):
        _run([NVCC, "-shared", "-cudart", "static"] + ARCH + ["-o", LIB] + objs + ["-ldl"], verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
