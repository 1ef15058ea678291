"""Build libcrmpm_b200.so (sm_100a) in place with nvcc.

    python cressim-mpm_b200/build.py [--debug]

The library is plain CUDA C++ with a C ABI (include/crmpm_b200.h); nothing here links against
torch.  Output: cressim-mpm_b200/libcrmpm_b200.so.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCES = ["csrc/mpm_kernels.cu", "csrc/capi.cu", "csrc/noalloc.cu", "csrc/sdf_builder.cu"]
OUT = os.path.join(HERE, "libcrmpm_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(HERE, s) for s in SOURCES]
    deps += [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc")) if f.endswith(".cuh")]
    deps.append(os.path.join(ROOT, "include", "crmpm_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    if not force and not needs_build():
        return OUT
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-fvisibility=hidden",
           "-I", os.path.join(ROOT, "include"), "-o", OUT + ".tmp"]
    cmd += extra or []
    cmd += [os.path.join(HERE, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    extra = ["-Xptxas", "-v"] if "-v" in sys.argv else []
    build(force=True, verbose=True, extra=extra)
