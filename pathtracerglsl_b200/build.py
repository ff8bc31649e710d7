"""Build recipe of the CUDA library ``pathtracerglsl_b200/libptx_rt.so`` (sm_100a).

nvcc cross-compiles without a GPU; the shared object is built in-tree so it travels
with the working tree.  ``-fmad=false`` keeps every product and sum rounded as written
(binary32 in the operation order of the reference's shader math).
"""
import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libptx_rt.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC,-O3", "-shared"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "**", "*.cu"), recursive=True) +
                  glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True) +
                  glob.glob(os.path.join(CSRC, "**", "*.cpp"), recursive=True) +
                  glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True) +
                  [os.path.join(ROOT, "include", "ptx_rt.h")])


def build(force=False, verbose=False):
    newest = max(os.path.getmtime(p) for p in sources())
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    units = [os.path.join(CSRC, "ptx_rt.cu")] + sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp")))
    cmd = [NVCC, *ARCH, *FLAGS, "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CSRC, "device"), *units,
           "-o", LIB + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stderr[-4000:])
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
