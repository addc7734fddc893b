"""Build libkerrsplat_b200.so in-tree with nvcc for sm_100a (B200)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libkerrsplat_b200.so")
SOURCES = ["ks_lib.cu"]
HEADERS = ["ks_elliptic.cuh", "ks_plan.cuh", "ks_march.cuh", "ks_dual.cuh", "ks_transfer.cuh", "ks_mixed.cuh", "ks_adjoint.cuh", "ks_spacetime.cuh", "ks_dft.cuh"]


def nvcc_command(out=LIB, extra=()):
    """FP32 division and square root take the hardware approximations (-prec-div=false,
    -prec-sqrt=false: a few ulp, inside the mixed path's 1e-4 budget; the coefficient fits divide
    often and the IEEE sequences cost them a quarter of their time). FP64 arithmetic is unaffected,
    denormals are kept."""
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    return [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
            "--use_fast_math" if os.environ.get("KS_FAST_MATH") else "-Xptxas=-O3",
            "-prec-div=false", "-prec-sqrt=false",
            "-shared", "-Xcompiler", "-fPIC", "-o", out] + list(extra) + [os.path.join(CSRC, s) for s in SOURCES]


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = SOURCES + HEADERS
    return any(os.path.getmtime(os.path.join(CSRC, d)) > t for d in deps) or \
        os.path.getmtime(os.path.join(HERE, "..", "include", "kerrsplat_b200.h")) > t


def build(force=False, verbose=True):
    """Compile the CUDA library if a source is newer than the .so (or `force`)."""
    if not force and not stale():
        return LIB
    cmd = nvcc_command()
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
