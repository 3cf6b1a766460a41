"""Build the sm_100a CUDA library in-tree: parallelkde.jl_b200/lib/libpkde_b200.so.

    python parallelkde.jl_b200/build.py [--force]

nvcc cross-compiles without a GPU.  The sources are compiled with FMA contraction left
on (the FFT and propagation arithmetic), while every operation whose rounding must match
the reference's CPU arithmetic is written with explicit __dadd_rn/__dmul_rn/__ddiv_rn
intrinsics, which are never contracted.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = ["pkde_ctx.cu", "pkde_binning.cu", "pkde_fft.cu", "pkde_step.cu", "pkde_engine.cu", "pkde_gradepro.cu"]
HDR = ["pkde_internal.cuh", "pkde_regfft.cuh", "pkde_step.cuh", os.path.join("..", "..", "include", "pkde_b200.h")]
OUT = os.path.join(HERE, "lib", "libpkde_b200.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def _newer(out, deps):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force=False, verbose=False):
    srcs = [os.path.join(HERE, "csrc", s) for s in SRC]
    deps = srcs + [os.path.join(HERE, "csrc", h) for h in HDR] + [os.path.abspath(__file__)]
    if not force and _newer(OUT, deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    if not os.path.exists(nvcc) and os.path.exists("/usr/local/cuda/bin/nvcc"):
        nvcc = "/usr/local/cuda/bin/nvcc" if nvcc == "nvcc" and not _which("nvcc") else nvcc
    cmd = [nvcc] + NVCC_FLAGS + ["-o", OUT] + srcs
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return OUT


def _which(x):
    for d in os.environ.get("PATH", "").split(os.pathsep):
        if os.path.exists(os.path.join(d, x)):
            return True
    return False


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
