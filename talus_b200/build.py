"""Builds libtalus_fem.so in-tree for sm_100a (nvcc -gencode arch=compute_100a,code=sm_100a)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = [os.path.join(HERE, "csrc", "tl_system.cu"), os.path.join(HERE, "csrc", "tl_noalloc.cu")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in ("tl_kernels.cuh", "tl_math.cuh", "tl_adjoint.cuh", "tl_sell.cuh",
                                                   "tl_sell_build.h", "tl_validate.h", "tl_floating.cuh",
                                                   "tl_factor.cuh", "tl_factor_host.h")] + [
    os.path.join(os.path.dirname(HERE), "include", "talus_fem.h")]
OUTPUT = os.path.join(HERE, "libtalus_fem.so")
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-pthread", "-Xptxas", "-v"]


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
    # each source compiles in its own nvcc process (in parallel), then one link
    objects = [os.path.splitext(src)[0] + ".o" for src in SOURCES]
    jobs = [subprocess.Popen([nvcc(), *NVCC_FLAGS, "-c", "-o", obj, src], stdout=subprocess.PIPE,
                             stderr=subprocess.PIPE, text=True) for src, obj in zip(SOURCES, objects)]
    logs = []
    failed = 0
    for job in jobs:
        out, err = job.communicate()
        logs.append(out + err)
        failed = failed or job.returncode
    if not failed:
        link = subprocess.run([nvcc(), "-shared", "-Xcompiler", "-pthread", "-gencode",
                               "arch=compute_100a,code=sm_100a", "-o", OUTPUT, *objects],
                              capture_output=True, text=True)
        logs.append(link.stdout + link.stderr)
        failed = link.returncode
    for obj in objects:
        if os.path.exists(obj):
            os.remove(obj)
    if verbose or failed:
        sys.stderr.write("".join(logs))
    if failed:
        raise RuntimeError(f"nvcc failed ({failed})")
    with open(os.path.join(HERE, "ptxas_info.txt"), "w") as f:
        f.write("".join(logs))
    return OUTPUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
