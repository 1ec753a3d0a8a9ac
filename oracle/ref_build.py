"""Builds the reference's own GPU routes into oracle/_ref/ (checker only).

Compiles the reference harness harness/primary/gpu_common_v0_6.cu (which
textually includes the Sparse-Seam v1.0 and Global-UF snapshots) unchanged,
from where it lies in the reference tree, for sm_100a, wrapped by
``ref_routes.cu`` and a small OpenCV stand-in header (``ref_shim/``).  One
library per reference tile size: T = 32 (the reference's reported setting)
and T = 64 (its source default).  Outputs go only to oracle/_ref/, which is
git-ignored but travels to the GPU host with the working tree.

The reference tree's location is given by the environment variable
``SS_REFERENCE_TREE`` (or ``--reference DIR`` on the command line); without
it nothing is built and the prebuilt libraries, if any, are used.  The GPU
host has no reference tree; it uses the prebuilt libraries.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
TILES = (32, 64)


def harness_dir(reference=None):
    """harness/primary of the reference tree, or None if no tree is given."""
    tree = reference or os.environ.get("SS_REFERENCE_TREE")
    return os.path.join(tree, "harness", "primary") if tree else None


def library(tile: int) -> str:
    return os.path.join(OUT, f"libssref_t{tile}.so")


def available(reference=None) -> bool:
    harness = harness_dir(reference)
    return bool(harness) and os.path.exists(
        os.path.join(harness, "gpu_common_v0_6.cu"))


def build(tile: int, force: bool = False, reference=None) -> str:
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
        "-I" + os.path.join(HERE, "ref_shim"), "-I" + harness_dir(reference),
        "-Xcompiler", "-fPIC", "-shared", "-w", "-o", tmp, src,
    ])
    os.replace(tmp, out)
    return out


def build_if_available(reference=None) -> list:
    if not available(reference):
        return [library(t) for t in TILES if os.path.exists(library(t))]
    return [build(t, reference=reference) for t in TILES]


if __name__ == "__main__":
    import argparse
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=None,
                        help="reference tree (default: $SS_REFERENCE_TREE)")
    cli = parser.parse_args()
    if not available(cli.reference):
        sys.exit("no reference tree: pass --reference DIR or set "
                 "SS_REFERENCE_TREE")
    print(build_if_available(cli.reference))
