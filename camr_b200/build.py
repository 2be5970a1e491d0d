"""Build libcamr_b200.so in-tree for sm_100a with nvcc.

-fmad=false keeps every product and sum separately rounded, which is what
makes the kernels reproduce the reference's CPU arithmetic bit for bit.
"""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib", "libcamr_b200.so")
SOURCES = ["hydro_kernels.cu", "level.cu", "peak.cu", "noalloc.cu", "batch.cu", "amr.cu",
           "adjoint.cu", "eb.cu", "fab_ops.cu", "io.cpp"]
HEADERS = ["camr_common.cuh", "hydro_point.cuh", "hydro_kernels.cuh", "level_point.cuh",
           "adjoint_point.cuh", "cell_point.cuh", "fastdiv.h", "rndiv.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "camr_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compile the CUDA sources into camr_b200/_lib/libcamr_b200.so."""
    if not force and not _stale():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = [nvcc(), *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"),
           *[os.path.join(CSRC, f) for f in SOURCES], "-o", OUT + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose=True))
