"""ctypes loader for the CPU oracle (test infrastructure only).

Only the tests, the smoke check and the benchmark's CPU-baseline leg import
this module.  It never stands in for the CUDA path: it is the checker.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

_LIB = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = _build.LIBRARY
        if not os.path.exists(path):
            path = _build.build()
        _LIB = ctypes.CDLL(path)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        for name in ("ss_oracle_floodfill", "ss_oracle_unionfind"):
            fn = getattr(_LIB, name)
            fn.argtypes = [u8p, ctypes.c_int, ctypes.c_int, ctypes.c_long,
                           u8p, u8p, ctypes.c_long]
            fn.restype = ctypes.c_int
        _LIB.ss_oracle_bands.argtypes = [
            u8p, ctypes.c_int, ctypes.c_int, ctypes.c_long, u8p, u8p,
            ctypes.c_long, ctypes.c_int]
        _LIB.ss_oracle_bands.restype = ctypes.c_int
        _LIB.ss_oracle_batch.argtypes = [
            ctypes.c_int, ctypes.POINTER(u8p), ctypes.POINTER(ctypes.c_int),
            ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_long),
            ctypes.POINTER(u8p), ctypes.POINTER(u8p),
            ctypes.POINTER(ctypes.c_long), ctypes.c_int]
        _LIB.ss_oracle_batch.restype = ctypes.c_int
        _LIB.ss_oracle_tile_fragments.argtypes = [
            u8p, ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_int,
            ctypes.POINTER(ctypes.c_uint16)]
        _LIB.ss_oracle_tile_fragments.restype = ctypes.c_int
        _LIB.ss_oracle_max_threads.argtypes = []
        _LIB.ss_oracle_max_threads.restype = ctypes.c_int
    return _LIB


def _u8(array: np.ndarray):
    return array.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


def _check_image(image: np.ndarray) -> np.ndarray:
    if image.dtype != np.uint8 or image.ndim != 2:
        raise ValueError("expected a 2-D uint8 image")
    if image.strides[1] != 1:
        image = np.ascontiguousarray(image)
    return image


def extrema(image: np.ndarray, method: str = "unionfind", threads: int = 0):
    """Returns (maxima, minima) as 0/255 uint8 arrays of the image's shape."""
    image = _check_image(image)
    h, w = image.shape
    maxima = np.empty((h, w), dtype=np.uint8)
    minima = np.empty((h, w), dtype=np.uint8)
    pitch = image.strides[0]
    if method == "floodfill":
        rc = lib().ss_oracle_floodfill(_u8(image), w, h, pitch, _u8(maxima),
                                       _u8(minima), w)
    elif method == "unionfind":
        rc = lib().ss_oracle_unionfind(_u8(image), w, h, pitch, _u8(maxima),
                                       _u8(minima), w)
    elif method == "bands":
        rc = lib().ss_oracle_bands(_u8(image), w, h, pitch, _u8(maxima),
                                   _u8(minima), w,
                                   threads or max_threads())
    else:
        raise ValueError(method)
    if rc != 0:
        raise RuntimeError(f"oracle {method} failed with {rc}")
    return maxima, minima


def extrema_batch(images, threads: int = 0):
    """Union-find route over a list of images, one image per thread."""
    images = [_check_image(im) for im in images]
    n = len(images)
    outs_max = [np.empty_like(im) for im in images]
    outs_min = [np.empty_like(im) for im in images]
    u8p = ctypes.POINTER(ctypes.c_uint8)
    ip = (u8p * n)(*[_u8(im) for im in images])
    mp = (u8p * n)(*[_u8(m) for m in outs_max])
    np_ = (u8p * n)(*[_u8(m) for m in outs_min])
    ws = (ctypes.c_int * n)(*[im.shape[1] for im in images])
    hs = (ctypes.c_int * n)(*[im.shape[0] for im in images])
    ps = (ctypes.c_long * n)(*[im.strides[0] for im in images])
    ops = (ctypes.c_long * n)(*[im.shape[1] for im in images])
    rc = lib().ss_oracle_batch(n, ip, ws, hs, ps, mp, np_, ops,
                               threads or max_threads())
    if rc != 0:
        raise RuntimeError(f"oracle batch failed with {rc}")
    return outs_max, outs_min


def tile_fragments(image: np.ndarray, tile: int) -> np.ndarray:
    """Per-tile count of tile-local flat zones with an equal outside neighbour."""
    image = _check_image(image)
    h, w = image.shape
    tx = (w + tile - 1) // tile
    ty = (h + tile - 1) // tile
    counts = np.zeros(tx * ty, dtype=np.uint16)
    rc = lib().ss_oracle_tile_fragments(
        _u8(image), w, h, image.strides[0], tile,
        counts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)))
    if rc != 0:
        raise RuntimeError(f"oracle tile_fragments failed with {rc}")
    return counts.reshape(ty, tx)


def max_threads() -> int:
    return int(lib().ss_oracle_max_threads())
