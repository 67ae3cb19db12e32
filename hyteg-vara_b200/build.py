"""Build the sm_100a shared library libhyteg_b200.so in-tree (no JIT cache).

    python hyteg-vara_b200/build.py [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = [os.path.join(HERE, "csrc", f) for f in ("hyb_capi.cu", "topology.cpp")]
DEPS = SRC + [os.path.join(HERE, "csrc", f) for f in ("hyb_device.cuh", "hyb_kernels.cuh", "hyb_program.cuh", "hyb_storage.inl", "hyb_launch.inl", "hyb_gmg.inl", "hyb_server.inl", "topology.hpp")] + \
    [os.path.join(os.path.dirname(HERE), "include", "hyteg_b200.h")]
OUT = os.path.join(HERE, "libhyteg_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
         "-shared", "-Xptxas", "-warn-spills"]


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in DEPS)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return OUT
    cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", OUT] + SRC
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
