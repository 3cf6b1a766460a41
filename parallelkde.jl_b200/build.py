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
SRC = ["pkde_ctx.cu", "pkde_binning.cu", "pkde_fft.cu", "pkde_step.cu", "pkde_engine.cu", "pkde_gradepro.cu",
       "pkde_serve.cu", "pkde_grid.cu"]
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
    if not _which(nvcc) and os.path.exists("/usr/local/cuda/bin/nvcc"):
        nvcc = "/usr/local/cuda/bin/nvcc"
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [nvcc] + compile_flags + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        return obj

    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, srcs))
    link = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT] + objs
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.check_call(link)
    return OUT


def _which(x):
    for d in os.environ.get("PATH", "").split(os.pathsep):
        if os.path.exists(os.path.join(d, x)):
            return True
    return False


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
