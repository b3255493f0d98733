"""Build librypath_cuda.so (the CUDA backend) in-tree with nvcc for sm_100a.

The library is the product: hand-written CUDA kernels plus the C ABI of
include/rypath_cuda.h.  ``build()`` recompiles only when a source is newer than the library.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librypath_cuda.so")
SOURCES = ["rp_host.cu"]
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith(".cuh"))
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if candidate and (os.path.isabs(candidate) and os.path.exists(candidate) or not os.path.isabs(candidate)):
            return candidate
    return "nvcc"


def command(output=LIB, extra=()):
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    return [nvcc(), ARCH, "-O3", "-std=c++20", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC",
            "-Xcompiler", "-ffp-contract=off", "-shared", "-o", output, *extra, *srcs]


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    built = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "rypath_cuda.h")]
    return any(os.path.getmtime(d) > built for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if force or stale():
        cmd = command()
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
