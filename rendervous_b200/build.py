"""Builds libvrt.so (sm_100a) in-tree with nvcc.

The shared library is written next to this file so it travels with the
package; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvrt.so")
SOURCES = ["vrt_api.cu", "vrt_transmittance.cu", "vrt_path.cu", "vrt_adjoint.cu", "vrt_wave.cu", "vrt_cache.cu",
           "vrt_noalloc.cu"]
HEADERS = ["vrt_device.cuh", "vrt_tracking.cuh", "vrt_params.h", "vrt_internal.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _inputs():
    paths = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    paths.append(os.path.join(HERE, "..", "include", "vrt.h"))
    return paths


STAMP = LIB + ".stamp"


def _digest() -> str:
    import hashlib
    h = hashlib.sha256()
    for p in _inputs():
        with open(p, "rb") as f:
            h.update(f.read())
    h.update(" ".join(NVCC_FLAGS).encode())
    return h.hexdigest()


def up_to_date() -> bool:
    """True when libvrt.so was built from exactly the current sources (content
    hash, so copies of the tree with fresh timestamps do not rebuild)."""
    if not (os.path.exists(LIB) and os.path.exists(STAMP)):
        return False
    with open(STAMP) as f:
        return f.read().strip() == _digest()


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> str:
    """Compile every .cu of csrc/ into one shared library with nvcc."""
    if not force and up_to_date():
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, *(extra_flags or []), "-shared", "-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("libvrt build failed:\n" + out.stdout + out.stderr)
    if not extra_flags:
        with open(STAMP, "w") as f:
            f.write(_digest())
    if verbose and out.stderr:
        print(out.stderr, file=sys.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra_flags=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)
    print(LIB)
