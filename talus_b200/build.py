"""Builds libtalus_fem.so in-tree for sm_100a (nvcc -gencode arch=compute_100a,code=sm_100a)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = [os.path.join(HERE, "csrc", "tl_system.cu"), os.path.join(HERE, "csrc", "tl_noalloc.cu")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in ("tl_kernels.cuh", "tl_math.cuh", "tl_adjoint.cuh", "tl_sell.cuh",
                                                   "tl_sell_build.h", "tl_validate.h")] + [
    os.path.join(os.path.dirname(HERE), "include", "talus_fem.h")]
OUTPUT = os.path.join(HERE, "libtalus_fem.so")
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-pthread", "-shared", "-Xptxas", "-v"]


def nvcc() -> str:
    home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = os.path.join(home, "bin", "nvcc")
    return path if os.path.exists(path) else "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(OUTPUT):
        return False
    built = os.path.getmtime(OUTPUT)
    return all(os.path.getmtime(p) <= built for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUTPUT
    cmd = [nvcc(), *NVCC_FLAGS, "-o", OUTPUT, *SOURCES]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode})")
    with open(os.path.join(HERE, "ptxas_info.txt"), "w") as f:
        f.write(res.stderr)
    return OUTPUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
