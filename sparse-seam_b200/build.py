"""Build recipe for the CUDA route library (sm_100a).

Compiles ``csrc/ss_route.cu`` (the route), ``csrc/ss_static.cu`` (its
zero-allocation form), ``csrc/ss_server.cu`` (the
serving loop), ``csrc/ss_pack.cu`` (compact mask transfer, host side with
OpenMP) and ``csrc/ss_image_io.cpp`` (PGM / PNG / BMP / JPEG / TIFF files, zlib) into ``libsparseseam.so`` next to this file with
nvcc.  The library has a plain C ABI (``include/sparse_seam.h``) and links the
CUDA runtime statically, so it loads into any process on the GPU host, with or
without PyTorch.
"""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
SOURCES = [os.path.join(HERE, "csrc", "ss_route.cu"),
           os.path.join(HERE, "csrc", "ss_static.cu"),
           os.path.join(HERE, "csrc", "ss_server.cu"),
           os.path.join(HERE, "csrc", "ss_pack.cu"),
           os.path.join(HERE, "csrc", "ss_image_io.cpp")]
DEPENDS = SOURCES + [
    os.path.join(HERE, "csrc", name)
    for name in ("ss_device.cuh", "ss_tile.cuh", "ss_rowscan.cuh",
                 "ss_runs.cuh", "ss_internal.h", "ss_pool.hpp",
                 "ss_percentile.hpp")
] + [os.path.join(INCLUDE, "sparse_seam.h")]
LIBRARY = os.path.join(HERE, "libsparseseam.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc",
                 shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def command(output: str, extra=()) -> list:
    return [
        nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17",
        "-I" + INCLUDE, "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
        "-shared", "-Xptxas", "-warn-spills",
        *extra, "-o", output, *SOURCES, "-lgomp", "-lz",
    ]


HARNESS_SOURCE = os.path.join(HERE, "csrc", "ss_harness.cpp")
HARNESS = os.path.join(HERE, "ss_harness")


def harness_command(output: str) -> list:
    """The command-line harness: host C++ over the C ABI, linked against
    the library next to it (rpath $ORIGIN)."""
    return [
        nvcc(), *ARCH, "-O2", "-std=c++17", "-I" + INCLUDE,
        "-I" + os.path.join(HERE, "csrc"), "-o", output,
        HARNESS_SOURCE, "-L" + HERE, "-lsparseseam",
        "-Xlinker", "-rpath,$ORIGIN",
    ]


def stale() -> bool:
    if not os.path.exists(LIBRARY) or not os.path.exists(HARNESS):
        return True
    built = min(os.path.getmtime(LIBRARY), os.path.getmtime(HARNESS))
    return any(os.path.getmtime(d) > built
               for d in DEPENDS + [HARNESS_SOURCE])


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIBRARY
    tmp = LIBRARY + ".tmp"
    extra = ["-Xptxas", "-v"] if verbose else []
    subprocess.check_call(command(tmp, extra))
    os.replace(tmp, LIBRARY)
    tmp = HARNESS + ".tmp"
    subprocess.check_call(harness_command(tmp))
    os.replace(tmp, HARNESS)
    return LIBRARY


if __name__ == "__main__":
    import sys
    print(build(force=True, verbose="-v" in sys.argv))
