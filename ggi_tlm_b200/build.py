"""Build the in-tree CUDA library libtlm_gpu.so for sm_100a with nvcc.

    python -m ggi_tlm_b200.build [--verbose]

The library is plain CUDA C++ with a C-ABI (include/tlm_gpu.h); it does not
link against PyTorch.  Output: ggi_tlm_b200/_lib/libtlm_gpu.so.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "libtlm_gpu.so")
SOURCES = [os.path.join(HERE, "csrc", "tlm_gpu.cu"), os.path.join(HERE, "csrc", "tlm_batch.cu")]
DEPS = SOURCES + [os.path.join(HERE, "csrc", "tlm_kernels.cuh"), os.path.join(ROOT, "include", "tlm_gpu.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def build(force: bool = False, verbose: bool = False) -> str:
    srcs = [s for s in SOURCES if os.path.exists(s)]
    deps = [d for d in DEPS if os.path.exists(d)]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp", *srcs]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    if verbose:
        sys.stderr.write(res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose="--verbose" in sys.argv))
