"""Build recipe for the sm_100a shared library (in-tree, next to this file).

    python -m aphid_git_b200.build          # -> aphid_git_b200/libaphid_gpu.so

nvcc cross-compiles for sm_100a without a GPU.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libaphid_gpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared"]


def sources():
    return sorted(os.path.join(SRC, f) for f in os.listdir(SRC)
                  if f.endswith((".cu", ".cuh", ".h")))


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    inc = os.path.join(os.path.dirname(HERE), "include")
    hdrs = [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return all(os.path.getmtime(s) <= t for s in sources() + hdrs)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    units = [os.path.join(SRC, f) for f in ("aphid_gpu.cu", "aphid_noalloc.cu", "aphid_unet.cu")]
    cmd = ["nvcc"] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", LIB] + units
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
