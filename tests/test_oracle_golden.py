"""Pins the CPU oracle to the reference's 206 golden cases (412 masks).

The golden masks were produced by MATLAB imregionalmax / imregionalmin with
8-connectivity (oracles/build_oracle_v0_1.m:109-110); the manifests give the
per-case mask pixel counts (oracles/*/oracle_manifest.csv).  Every oracle route
must reproduce every mask exactly, and the manifest counts, before any GPU
result is compared against the oracle.
"""
import numpy as np
import pytest

import oracle


def test_fixture_inventory(golden_cases):
    suites = {}
    for c in golden_cases:
        suites[c.suite] = suites.get(c.suite, 0) + 1
    assert suites == {
        "oracle_v0_1": 34,
        "oracle_v0_2_fuzz": 160,
        "oracle_v0_3_sparse_seam_adversarial": 12,
    }


def test_golden_masks_match_manifest(golden_cases):
    for c in golden_cases:
        assert int((c.maxima != 0).sum()) == c.manifest_max, c
        assert int((c.minima != 0).sum()) == c.manifest_min, c


@pytest.mark.parametrize("method", ["floodfill", "unionfind", "bands"])
def test_oracle_routes_reproduce_golden(golden_cases, method):
    for c in golden_cases:
        mx, mn = oracle.extrema(c.image, method=method, threads=3)
        assert np.array_equal(mx, c.maxima), (method, c)
        assert np.array_equal(mn, c.minima), (method, c)


def test_oracle_batch_reproduces_golden(golden_cases):
    images = [c.image for c in golden_cases]
    maxs, mins = oracle.extrema_batch(images, threads=4)
    for c, mx, mn in zip(golden_cases, maxs, mins):
        assert np.array_equal(mx, c.maxima), c
        assert np.array_equal(mn, c.minima), c


def test_oracle_respects_pitch():
    rng = np.random.default_rng(7)
    base = (rng.integers(0, 256, size=(37, 53)) >> 5 << 5).astype(np.uint8)
    padded = np.full((37, 64), 99, dtype=np.uint8)
    padded[:, :53] = base
    view = padded[:, :53]
    for method in ("floodfill", "unionfind", "bands"):
        a = oracle.extrema(base, method=method)
        b = oracle.extrema(view, method=method)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_oracle_routes_agree_on_random_images():
    rng = np.random.default_rng(20260728)
    for trial in range(60):
        h = int(rng.integers(1, 90))
        w = int(rng.integers(1, 90))
        levels = int(rng.choice([2, 3, 4, 8, 16, 256]))
        img = rng.integers(0, levels, size=(h, w)).astype(np.uint8)
        ref = oracle.extrema(img, method="floodfill")
        for method in ("unionfind", "bands"):
            got = oracle.extrema(img, method=method, threads=5)
            assert np.array_equal(got[0], ref[0]), (trial, method)
            assert np.array_equal(got[1], ref[1]), (trial, method)


def test_tile_fragment_counts_small_cases():
    # A constant 64x64 image at T=32: every tile's single zone touches a seam.
    img = np.full((64, 64), 5, dtype=np.uint8)
    assert oracle.tile_fragments(img, 32).tolist() == [[1, 1], [1, 1]]
    # One tile only: nothing lies outside it inside the image.
    assert oracle.tile_fragments(img, 64).tolist() == [[0]]
    # Checkerboard: the two diagonal classes both cross every seam.
    yy, xx = np.mgrid[0:64, 0:64]
    cb = (((xx + yy) & 1) * 200).astype(np.uint8)
    assert oracle.tile_fragments(cb, 32).tolist() == [[2, 2], [2, 2]]
