"""Builds the reference's own GPU routes into oracle/_ref/ (checker only).

Compiles the reference harness harness/primary/gpu_common_v0_6.cu (which
textually includes the Sparse-Seam v1.0 and Global-UF snapshots) unchanged,
from where it lies in the reference tree, for sm_100a, wrapped by
``ref_routes.cu`` and a small OpenCV stand-in header (``ref_shim/``).  One
library per reference tile size: T = 32 (the reference's reported setting)
and T = 64 (its source default).  Outputs go only to oracle/_ref/, which is
git-ignored but travels to the GPU host with the working tree.

The GPU host has no reference tree; it uses the prebuilt libraries.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
REFERENCE = os.environ.get("SS_REFERENCE_TREE", "/root/reference")
HARNESS = os.path.join(REFERENCE, "harness", "primary")
TILES = (32, 64)


def library(tile: int) -> str:
    return os.path.join(OUT, f"libssref_t{tile}.so")


def available() -> bool:
    return os.path.exists(os.path.join(HARNESS, "gpu_common_v0_6.cu"))


def build(tile: int, force: bool = False) -> str:
    out = library(tile)
    src = os.path.join(HERE, "ref_routes.cu")
    if not force and os.path.exists(out) and \
            os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    os.makedirs(OUT, exist_ok=True)
    from importlib import import_module
    nvcc = import_module("sparse-seam_b200.build").nvcc()
    tmp = out + ".tmp"
    subprocess.check_call([
        nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
        "-std=c++17", f"-DSS_TILE={tile}", "-DSS_CLASSIFY_VARIANT=1",
        "-I" + os.path.join(HERE, "ref_shim"), "-I" + HARNESS,
        "-Xcompiler", "-fPIC", "-shared", "-w", "-o", tmp, src,
    ])
    os.replace(tmp, out)
    return out


def build_if_available() -> list:
    if not available():
        return [library(t) for t in TILES if os.path.exists(library(t))]
    return [build(t) for t in TILES]


if __name__ == "__main__":
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    print(build_if_available())
