"""Build recipe for the CPU oracle (test infrastructure).

Compiles ``ss_oracle.c`` into ``oracle/liboracle.so`` with gcc and OpenMP.
The shared object is git-ignored but travels with the working tree, so the
GPU-side tests and the benchmark's CPU-baseline leg load the prebuilt file.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCE = os.path.join(HERE, "ss_oracle.c")
LIBRARY = os.path.join(HERE, "liboracle.so")


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIBRARY) and \
            os.path.getmtime(LIBRARY) >= os.path.getmtime(SOURCE):
        return LIBRARY
    tmp = LIBRARY + ".tmp"
    subprocess.check_call([
        "gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared",
        "-Wall", "-Wextra", "-o", tmp, SOURCE,
    ])
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force=True))
