"""Seeded synthetic image generators for the route's workloads.

The reference timed public corpora (DIV2K 2040x1356 images, BSDS500 481x321,
BBBC038 distance maps) that are not available here; these generators stand in
for them with the same sizes and value structure:

  uniform_q16         i.i.d. uniform 0..255 quantised to 16 levels (v>>4<<4)
  constant            one value everywhere
  smooth_noise        sum of three Gaussian-filtered white-noise fields
                      (sigma 1, 4, 16 px; weights 0.2, 0.3, 0.5), min-max
                      normalised to 0..255, plus uniform integer noise in
                      [-2, 2], clamped -- natural-image-like.  Each filtered
                      field is scaled to unit standard deviation before the
                      weights apply; otherwise filtering alone would shrink
                      the sigma-4 and sigma-16 fields to a few percent of the
                      sigma-1 field and the sum would be close to white noise
  quantize            re-quantisation to L gray levels with the reference's
                      rule bin = (v*L) >> 8, out = round(bin*255/(L-1))
                      (harness/quantization_and_scaling/
                      gpu_common_quant_v0_7.cu:479-494)
  ellipse_edt         20-200 random ellipses (semi-axes 8-60 px, random
                      rotation), Euclidean distance transform of the union,
                      floored and clamped to 0..255 (large flat ridges; stands
                      in for the BBBC038 distance maps,
                      datasets/bbbc038_distance/
                      derive_bbbc038_distance_markers_v0_2.py:15-59)
  serpentine / spiral 1-px constant-valued paths on a background one gray
                      level lower, crossing every tile seam
  blocks              8x8 random-valued blocks aligned to the tile grid or
                      shifted by `offset` (the alignment control,
                      datasets/synthetic_alignment_control/
                      generate_scaling_suite_v0_2.cu:54-67)
  checkerboard        two-level checkerboard of a given cell size
  uneven_batch        images with width and height log-uniform in 64..1024,
                      50% smooth noise, 25% uniform-quantised (levels 2..256),
                      25% plateau maps

Everything is numpy on the host except smooth_noise, which uses torch so that
large corpora can be generated on the GPU (on either device the result is a
deterministic function of the seed).
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np


def uniform_q16(height: int, width: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = rng.integers(0, 256, size=(height, width), dtype=np.int32)
    return ((v >> 4) << 4).astype(np.uint8)


def constant(height: int, width: int, value: int = 128) -> np.ndarray:
    return np.full((height, width), value, dtype=np.uint8)


def quantize(image: np.ndarray, levels: int) -> np.ndarray:
    if levels >= 256:
        return image.copy()
    if levels < 2:
        raise ValueError("levels must be >= 2")
    b = (image.astype(np.int32) * levels) >> 8
    return ((b * 255 + (levels - 1) // 2) // (levels - 1)).astype(np.uint8)


def _gaussian_taps(sigma: float):
    import torch
    radius = max(1, int(math.ceil(4.0 * sigma)))
    x = torch.arange(-radius, radius + 1, dtype=torch.float32)
    k = torch.exp(-0.5 * (x / sigma) ** 2)
    return k / k.sum(), radius


def smooth_noise(height: int, width: int, seed: int = 0, device="cpu"):
    """Natural-image-like field; returns a torch uint8 tensor on `device`."""
    import torch
    import torch.nn.functional as F
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    acc = torch.zeros((height, width), dtype=torch.float32, device=device)
    for sigma, weight in ((1.0, 0.2), (4.0, 0.3), (16.0, 0.5)):
        noise = torch.randn((1, 1, height, width), generator=gen,
                            device=device, dtype=torch.float32)
        taps, r = _gaussian_taps(sigma)
        taps = taps.to(device)
        x = F.pad(noise, (r, r, 0, 0), mode="replicate")
        x = F.conv2d(x, taps.view(1, 1, 1, -1))
        x = F.pad(x, (0, 0, r, r), mode="replicate")
        x = F.conv2d(x, taps.view(1, 1, -1, 1))[0, 0]
        acc += weight * x / torch.clamp(x.std(), min=1e-12)
    lo, hi = acc.min(), acc.max()
    scaled = (acc - lo) * (255.0 / torch.clamp(hi - lo, min=1e-12))
    jitter = torch.randint(-2, 3, (height, width), generator=gen,
                           device=device, dtype=torch.int32)
    out = torch.clamp(torch.round(scaled).to(torch.int32) + jitter, 0, 255)
    return out.to(torch.uint8)


def smooth_noise_np(height: int, width: int, seed: int = 0) -> np.ndarray:
    return smooth_noise(height, width, seed, device="cpu").numpy()


def ellipse_edt(height: int = 1024, width: int = 1024,
                seed: int = 0) -> np.ndarray:
    from scipy import ndimage
    rng = np.random.default_rng(seed)
    mask = np.zeros((height, width), dtype=bool)
    for _ in range(int(rng.integers(20, 201))):
        cy = rng.uniform(0, height)
        cx = rng.uniform(0, width)
        a = rng.uniform(8, 60)
        b = rng.uniform(8, 60)
        t = rng.uniform(0, math.pi)
        y0, y1 = int(max(0, cy - 61)), int(min(height, cy + 62))
        x0, x1 = int(max(0, cx - 61)), int(min(width, cx + 62))
        dy = np.arange(y0, y1)[:, None] - cy
        dx = np.arange(x0, x1)[None, :] - cx
        u = dx * math.cos(t) + dy * math.sin(t)
        v = -dx * math.sin(t) + dy * math.cos(t)
        mask[y0:y1, x0:x1] |= (u / a) ** 2 + (v / b) ** 2 <= 1.0
    edt = ndimage.distance_transform_edt(mask)
    return np.clip(np.floor(edt), 0, 255).astype(np.uint8)


def serpentine(height: int = 1024, width: int = 1024, value: int = 101,
               period: int = 6) -> np.ndarray:
    """1-px horizontal runs joined alternately at the left / right end."""
    img = np.full((height, width), value - 1, dtype=np.uint8)
    rows = list(range(1, height - 1, period))
    for i, y in enumerate(rows):
        img[y, 1:width - 1] = value
        if i + 1 < len(rows):
            x = width - 2 if i % 2 == 0 else 1
            img[y:rows[i + 1] + 1, x] = value
    return img


def spiral(height: int = 1024, width: int = 1024, value: int = 77,
           gap: int = 3) -> np.ndarray:
    """A 1-px rectangular spiral on a background one level lower."""
    img = np.full((height, width), value - 1, dtype=np.uint8)
    top, left, bottom, right = 1, 1, height - 2, width - 2
    while top <= bottom and left <= right:
        img[top, left:right + 1] = value
        img[top:bottom + 1, right] = value
        if bottom - top >= gap:
            img[bottom, left:right + 1] = value
        if right - left >= gap:
            img[top + gap:bottom + 1, left] = value
        top += gap
        left += gap
        bottom -= gap
        right -= gap
        if top <= bottom and left - gap >= 0:
            img[top, left - gap:left + 1] = value
    return img


def blocks(height: int = 1024, width: int = 1024, block: int = 8,
           offset: int = 0, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    gy = (np.arange(height) + offset) // block
    gx = (np.arange(width) + offset) // block
    vals = rng.integers(0, 256, size=(gy.max() + 1, gx.max() + 1),
                        dtype=np.int32).astype(np.uint8)
    return vals[gy[:, None], gx[None, :]]


def checkerboard(height: int = 1024, width: int = 1024, cell: int = 1,
                 low: int = 0, high: int = 255) -> np.ndarray:
    yy, xx = np.mgrid[0:height, 0:width]
    on = ((yy // cell) + (xx // cell)) & 1
    return np.where(on, high, low).astype(np.uint8)


def plateau_map(height: int, width: int, seed: int = 0) -> np.ndarray:
    """One of the plateau- and seam-heavy families, chosen by the seed."""
    rng = np.random.default_rng(seed)
    kind = int(rng.integers(0, 4))
    if kind == 0:
        return ellipse_edt(height, width, seed)
    if kind == 1:
        return serpentine(height, width, int(rng.integers(1, 256)),
                          int(rng.integers(3, 9)))
    if kind == 2:
        return blocks(height, width, 8, int(rng.integers(0, 2)) * 16, seed)
    return checkerboard(height, width, int(rng.choice([1, 3, 17])))


def uneven_sizes(count: int, seed: int = 0, lo: int = 64,
                 hi: int = 1024) -> List[Tuple[int, int]]:
    rng = np.random.default_rng(seed)
    logs = rng.uniform(math.log(lo), math.log(hi), size=(count, 2))
    dims = np.clip(np.round(np.exp(logs)), lo, hi).astype(int)
    return [(int(h), int(w)) for h, w in dims]


def uneven_batch(count: int, seed: int = 0, lo: int = 64, hi: int = 1024,
                 device="cpu"):
    """Mixed-generator batch as a list of torch uint8 tensors on `device`."""
    import torch
    rng = np.random.default_rng(seed + 1)
    out = []
    for i, (h, w) in enumerate(uneven_sizes(count, seed, lo, hi)):
        u = rng.uniform()
        s = seed * 100003 + i
        if u < 0.5:
            out.append(smooth_noise(h, w, s, device=device))
            continue
        if u < 0.75:
            levels = int(rng.integers(2, 257))
            r2 = np.random.default_rng(s)
            img = quantize(r2.integers(0, 256, size=(h, w)).astype(np.uint8),
                           levels)
        else:
            img = plateau_map(h, w, s)
        out.append(torch.from_numpy(img).to(device))
    return out
