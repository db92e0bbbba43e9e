"""In-tree build of libgrhd_b200.so for sm_100a (nvcc, no JIT cache).

Each CUDA source compiles to its own object under grdzhadzha_b200/_build/
(in parallel; an object is rebuilt when its source or any header is newer),
then nvcc links the shared library."""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
CSRC = os.path.join(_HERE, "csrc")
BUILD_DIR = os.path.join(_HERE, "_build")
SOURCES = ["grhd_kernels.cu", "grhd_initial_data.cu", "grhd_capi.cu",
           "grhd_ensemble.cu", "grhd_adjoint.cu", "grhd_kitp.cu",
           "grhd_io.cu"]
OUTPUT = os.path.join(_HERE, "libgrhd_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo",
                     "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
          if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(_ROOT, "include", "grhd_b200.h"))
    return hs


def _obj(src: str) -> str:
    return os.path.join(BUILD_DIR, src[:-3] + ".o")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def needs_rebuild() -> bool:
    deps = [os.path.join(CSRC, s) for s in SOURCES] + _headers()
    return _stale(OUTPUT, deps)


def _compile(src: str, verbose: bool) -> None:
    cmd = [nvcc()] + NVCC_FLAGS + [
        "-I", os.path.join(_ROOT, "include"), "-I", CSRC,
        "-c", os.path.join(CSRC, src), "-o", _obj(src)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_rebuild():
        return OUTPUT
    os.makedirs(BUILD_DIR, exist_ok=True)
    hs = _headers()
    todo = [s for s in SOURCES
            if force or _stale(_obj(s), [os.path.join(CSRC, s)] + hs)]
    with cf.ThreadPoolExecutor(max_workers=max(1, len(todo))) as ex:
        for f in [ex.submit(_compile, s, verbose) for s in todo]:
            f.result()
    cmd = [nvcc()] + ARCH + ["-shared", "-o", OUTPUT] + [
        _obj(s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return OUTPUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
