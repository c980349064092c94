"""Builds libdspbr_cuda.so in-tree (dspbr-pt_b200/dspbr/) for sm_100a.

nvcc cross-compiles without a GPU.  The library is plain C ABI
(include/dspbr.h); nothing here links against torch.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "dspbr", "libdspbr_cuda.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["api.cu", "engine.cu", "server.cu", "display.cu", "kernels.cu", "ibl.cu", "ibl_noalloc.cu", "bvh_build.cpp", "bvh_wide.cpp", "bvh_gpu.cu"]


# files whose arithmetic must round every operation like the shader it restates
NO_FMA = {"display.cu"}


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "dspbr.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not stale():
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC, "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
               "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        if os.path.basename(src) in NO_FMA:
            cmd.insert(1, "-fmad=false")
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC, "-shared", *ARCH, "-o", OUT, *objs, "-lpthread"]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
