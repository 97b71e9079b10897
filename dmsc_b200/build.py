"""Builds the CUDA library ``dmsc_b200/libdmsc_b200.so`` for sm_100a.

One nvcc invocation compiles ``csrc/dmsc_b200.cu`` (which includes the other
kernel sources) and ``csrc/noalloc.cu`` into a position-independent shared
library exporting the C ABI declared in ``include/dmsc_b200.h``. The library is built in-tree so that it
travels with the repository snapshot; it is loaded with ctypes.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libdmsc_b200.so")
SRC_DIR = os.path.join(HERE, "csrc")
MAIN = os.path.join(SRC_DIR, "dmsc_b200.cu")
UNITS = [MAIN, os.path.join(SRC_DIR, "noalloc.cu")]  # translation units of the library
HEADER = os.path.join(ROOT, "include", "dmsc_b200.h")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def sources() -> list[str]:
    return sorted(os.path.join(SRC_DIR, f) for f in os.listdir(SRC_DIR) if f.endswith((".cu", ".cuh"))) + [HEADER]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [_nvcc(), *NVCC_FLAGS, *(extra or []), "-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp", *UNITS]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, extra=["-Xptxas", "-v"] if "-v" in sys.argv else None))
