"""Builds the in-tree shared library gr-athena_b200/_build/libz4c_b200.so.

The CUDA sources are compiled for sm_100a only (B200).  -fmad=false keeps
every multiply and add of the device code separately rounded, as the
reference CPU build (-ffp-contract=off) does; the host code (the extraction
spheres' tables) gets -ffp-contract=off itself.  The differentiated path
(z4c_adjoint.cu) is bound to no reference rounding and contracts
multiply-adds.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libz4c_b200.so")
SOURCES = ["z4c_kernels.cu", "z4c_capi.cu", "z4c_refine.cu", "z4c_noalloc.cu", "z4c_wave.cu",
           "z4c_restart.cu", "z4c_multilevel.cu", "z4c_adjoint.cu", "z4c_fast.cu"]
# per-file replacements of the default flags: the adjoint and the contracted
# right-hand side are built with floating-point contraction
FILE_FLAGS = {"z4c_adjoint.cu": {"-fmad=false": "-fmad=true"},
              "z4c_fast.cu": {"-fmad=false": "-fmad=true"}}
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "-Xcompiler", "-ffp-contract=off"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "z4c_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
        flags = [FILE_FLAGS.get(src, {}).get(f, f) for f in FLAGS]
        cmd = [NVCC, *flags, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
