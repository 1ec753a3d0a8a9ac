"""Parity with the reference's own GPU routes, compiled unchanged for sm_100a.

oracle/_ref/libssref_t{32,64}.so hold the reference harness
(harness/primary/gpu_common_v0_6.cu with the Sparse-Seam v1.0 and Global-UF
snapshots) built by oracle/ref_build.py.  The product's masks must equal the
reference routes' masks byte for byte, and the product's fragment statistics
must equal the reference's tile_fragment_counts sum at the same tile size.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle
from conftest import ROOT, package

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref")


def ref_lib(tile):
    path = os.path.join(REF, f"libssref_t{tile}.so")
    if not os.path.exists(path):
        pytest.skip(f"{path} not built (needs the reference tree at build time)")
    lib = ctypes.CDLL(path)
    u8 = ctypes.POINTER(ctypes.c_uint8)
    d = ctypes.POINTER(ctypes.c_double)
    lib.ssref_sparse_seam.argtypes = [u8, ctypes.c_int, ctypes.c_int, u8, u8,
                                      ctypes.c_int, ctypes.c_int, d, d,
                                      ctypes.POINTER(ctypes.c_longlong)]
    lib.ssref_global_uf.argtypes = [u8, ctypes.c_int, ctypes.c_int, u8, u8,
                                    ctypes.c_int, ctypes.c_int, d, d]
    return lib


def reference_masks(lib, img, route):
    h, w = img.shape
    img = np.ascontiguousarray(img)
    mx = np.zeros_like(img)
    mn = np.zeros_like(img)
    u8 = ctypes.POINTER(ctypes.c_uint8)
    ms = ctypes.c_double()
    h2h = ctypes.c_double()
    if route == "sparse":
        frag = ctypes.c_longlong()
        rc = lib.ssref_sparse_seam(img.ctypes.data_as(u8), w, h,
                                   mx.ctypes.data_as(u8), mn.ctypes.data_as(u8),
                                   0, 1, ctypes.byref(ms), ctypes.byref(h2h),
                                   ctypes.byref(frag))
        assert rc == 0
        return mx, mn, int(frag.value)
    rc = lib.ssref_global_uf(img.ctypes.data_as(u8), w, h,
                             mx.ctypes.data_as(u8), mn.ctypes.data_as(u8),
                             0, 1, ctypes.byref(ms), ctypes.byref(h2h))
    assert rc == 0
    return mx, mn, None


def images():
    import importlib
    synth = importlib.import_module("sparse-seam_b200.synth")
    rng = np.random.default_rng(3)
    out = [synth.uniform_q16(512, 512, 0), synth.constant(512, 512, 128),
           synth.smooth_noise_np(321, 481, 1),
           synth.quantize(synth.smooth_noise_np(321, 481, 2), 4),
           synth.checkerboard(257, 193, 3), synth.serpentine(300, 260)]
    for _ in range(6):
        h, w = int(rng.integers(20, 260)), int(rng.integers(20, 260))
        out.append(rng.integers(0, int(rng.choice([2, 4, 16])),
                                size=(h, w)).astype(np.uint8))
    return out


@pytest.mark.parametrize("tile,warps", [(32, -2), (32, -4), (32, 8), (64, -4),
                                        (64, 16)])
def test_product_matches_reference_routes(tile, warps):
    pkg = package()
    lib = ref_lib(tile)
    before = pkg.get_kernel_config(tile)
    pkg.set_kernel_config(tile, warps)
    try:
        check_against_reference(pkg, lib, tile, warps)
    finally:
        pkg.set_kernel_config(tile, before)


def check_against_reference(pkg, lib, tile, warps):
    for img in images():
        h, w = img.shape
        d = torch.from_numpy(img).cuda()
        ws = pkg.Workspace.for_image(w, h, tile)
        mx, mn = pkg.extrema(d, tile=tile, workspace=ws)
        stats = ws.read_status()
        got = (mx.cpu().numpy(), mn.cpu().numpy())
        smx, smn, sfrag = reference_masks(lib, img, "sparse")
        gmx, gmn, _ = reference_masks(lib, img, "globaluf")
        assert np.array_equal(got[0], smx) and np.array_equal(got[1], smn)
        assert np.array_equal(got[0], gmx) and np.array_equal(got[1], gmn)
        assert sfrag == int(oracle.tile_fragments(img, tile).sum())
        if warps > 0:
            assert stats.active_fragments == sfrag
        else:
            assert stats.active_fragments <= sfrag
