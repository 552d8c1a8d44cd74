"""Build the engine library in-tree: ``python -m gridsim_b200.build``.

One nvcc invocation for sm_100a (Blackwell B200); the shared library lands next to this file so it
travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = [os.path.join(HERE, "csrc", f) for f in ("gs_engine.cu", "gs_host.cpp", "gs_symbolic.cpp", "gs_dc.cpp",
                                                "gs_topology.cpp")]
OUT = os.path.join(HERE, "libgridsim_b200.so")
DEPS = SRC + [os.path.join(HERE, "csrc", f) for f in ("gs_internal.h", "gs_host.h", "gs_kernels.cuh", "gs_multi.cuh", "gs_serve.cuh", "gs_cluster.cuh", "gs_paired.cuh", "gs_pivot.cuh")] + [
    os.path.join(os.path.dirname(HERE), "include", "gridsim_b200.h")]


def nvcc() -> str:
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if p and (os.path.isabs(p) and os.path.exists(p) or not os.path.isabs(p)):
            return p
    return "nvcc"


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(d) for d in DEPS):
        return OUT
    cmd = [nvcc(), "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3",
           "-Xcompiler", "-fPIC", "-shared", "-o", OUT] + SRC
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
