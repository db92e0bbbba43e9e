"""In-tree build of libgrhd_b200.so for sm_100a (nvcc, no JIT cache)."""
from __future__ import annotations

import os
import subprocess
import sys

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
CSRC = os.path.join(_HERE, "csrc")
SOURCES = ["grhd_kernels.cu", "grhd_initial_data.cu", "grhd_capi.cu",
           "grhd_ensemble.cu", "grhd_adjoint.cu", "grhd_kitp.cu",
           "grhd_io.cu"]
OUTPUT = os.path.join(_HERE, "libgrhd_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def needs_rebuild() -> bool:
    if not os.path.exists(OUTPUT):
        return True
    t = os.path.getmtime(OUTPUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(_ROOT, "include", "grhd_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_rebuild():
        return OUTPUT
    cmd = [nvcc()] + NVCC_FLAGS + [
        "-I", os.path.join(_ROOT, "include"), "-I", CSRC,
        "-o", OUTPUT] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return OUTPUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
