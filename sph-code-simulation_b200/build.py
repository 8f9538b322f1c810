"""Build recipe for libsphgpu.so (sm_100a) — used by __graft_entry__.build().

Compiles every CUDA source under csrc/ with nvcc for sm_100a and links them,
with the host-side sample generators, into an in-tree shared library
``sph-code-simulation_b200/libsphgpu.so``.  Files whose results must match
the reference bit-for-bit (tree build, neighbour walks, gravity walk,
integration) are compiled with ``-fmad=false``: the reference is built for
x86-64 without FMA contraction.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsphgpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
EXACT = {"tree.cu", "walk.cu", "gravity.cu", "integrate.cu", "noalloc.cu", "relax.cu", "srgsph.cu"}
SOURCES = ["scan_sort.cu", "tree.cu", "walk.cu", "pre.cu", "force.cu", "gravity.cu", "gravity_mixed.cu", "flist.cu",
           "integrate.cu", "mlp.cu", "capi.cu", "noalloc.cu", "relax.cu", "srgsph.cu", "recheck.cu"]
HOST_SOURCES = ["samples.cpp", "csv.cpp"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _newer(src_files, out) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in src_files)


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(ROOT, "include", "sphgpu.h"))
    cmds = []
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        flags = list(NVFLAGS)
        if s in EXACT:
            flags.append("-fmad=false")
        if _newer([src] + headers, obj):
            cmds.append([nvcc] + ARCH + flags + ["-c", src, "-o", obj])
    for s in HOST_SOURCES:
        src = os.path.join(HOST, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if _newer([src] + headers, obj):
            cmds.append(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off",
                         "-I" + os.path.join(ROOT, "include"), "-c", src, "-o", obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr.strip():
            print(r.stderr, flush=True)

    with ThreadPoolExecutor(max_workers=jobs) as ex:
        list(ex.map(run, cmds))
    if cmds or _newer(objs, LIB):
        run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lpthread"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
