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
SOURCES = ["vrt_api.cu", "vrt_transmittance.cu", "vrt_path.cu", "vrt_adjoint.cu", "vrt_wave.cu", "vrt_wave_ds.cu",
           "vrt_cache.cu", "vrt_noalloc.cu", "vrt_collision.cu", "vrt_fp64.cu", "vrt_wave_drt.cu", "vrt_wave_sps.cu"]
HEADERS = ["vrt_device.cuh", "vrt_tracking.cuh", "vrt_params.h", "vrt_internal.h", "vrt_wave.cuh"]

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
    h.update(repr(sorted(PER_FILE_FLAGS.items())).encode())
    return h.hexdigest()


def up_to_date() -> bool:
    """True when libvrt.so was built from exactly the current sources (content
    hash, so copies of the tree with fresh timestamps do not rebuild)."""
    if not (os.path.exists(LIB) and os.path.exists(STAMP)):
        return False
    with open(STAMP) as f:
        return f.read().strip() == _digest()


# Files whose kernels round every operation on its own (no a*b+c contracted
# into an FMA).  vrt_wave_ds.cu: the NEE_DS primal and replay walks are
# separate kernels that must retrace the same path bit for bit.  vrt_path.cu:
# the position samplers of the DRT / DRTQ / SPS adjoints draw once per
# majorant-brick crossing, so a face distance one ulp off changes how many
# draws a sample takes; rounding as the CPU restatement does keeps them on the
# same paths.  vrt_collision.cu and vrt_fp64.cu: the collision integrators and
# the FP64 tracer follow the CPU restatement's rounding the same way.
# vrt_wave_drt.cu, vrt_wave_sps.cu: the DRT and SPS wavefronts' primals take the
# sequential forms' paths.
PER_FILE_FLAGS = {"vrt_wave_ds.cu": ["-fmad=false"], "vrt_path.cu": ["-fmad=false"], "vrt_collision.cu": ["-fmad=false"],
                  "vrt_fp64.cu": ["-fmad=false"], "vrt_wave_drt.cu": ["-fmad=false"],
                  "vrt_wave_sps.cu": ["-fmad=false"]}
OBJ_DIR = os.path.join(HERE, "_build")


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> str:
    """Compile every .cu of csrc/ (in parallel, one object each) and link them
    into one shared library with nvcc."""
    if not force and up_to_date():
        return LIB
    digest = _digest()  # of the sources as compiled (a file edited during the build leaves the stamp stale)
    os.makedirs(OBJ_DIR, exist_ok=True)
    procs = []
    for src in SOURCES:
        obj = os.path.join(OBJ_DIR, src[:-3] + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, *PER_FILE_FLAGS.get(src, []), *(extra_flags or []), "-c",
               os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, obj, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    errors = []
    for src, obj, proc in procs:
        out, err = proc.communicate()
        if proc.returncode != 0:
            errors.append(f"{src}:\n{out}{err}")
        elif verbose and err:
            print(err, file=sys.stderr)
    if errors:
        raise RuntimeError("libvrt build failed:\n" + "\n".join(errors))
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB] + [o for _, o, _ in procs]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("libvrt link failed:\n" + out.stdout + out.stderr)
    if not extra_flags:
        with open(STAMP, "w") as f:
            f.write(digest)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra_flags=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)
    print(LIB)
