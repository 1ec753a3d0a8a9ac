"""The zero-allocation entry point against the workspace entry point.

ss_extrema_static_scratch serves callers that cannot allocate device memory
(an allocator callback, a latency-critical loop, a plug-in whose host owns
every device allocation): its scratch is a fixed array inside the library.
Its masks must equal those of ss_extrema (bytes, so exactly) on two calls in
a row; once warmed up, further calls must allocate no device memory; its
status read-back must report the calls' outcome; the first call in a fresh
process (which sets the array up) must work too; and images beyond the
array's capacity are refused without touching the outputs.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, package

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def call_static(lib, image, tile, maxima, minima):
    h, w = image.shape
    stream = torch.cuda.current_stream().cuda_stream
    return lib.ss_extrema_static_scratch(
        image.data_ptr(), w, h, image.stride(0), tile, maxima.data_ptr(),
        minima.data_ptr(), maxima.stride(0), ctypes.c_void_p(stream))


def read_static_status(pkg, lib):
    stats = pkg.Stats()
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.ss_static_scratch_read_status(ctypes.c_void_p(stream),
                                           ctypes.byref(stats))
    return rc, stats


def cases():
    import importlib
    synth = importlib.import_module("sparse-seam_b200.synth")
    rng = np.random.default_rng(17)
    return [
        (synth.smooth_noise(1356, 2040, seed=5, device="cuda"), 32),
        (torch.from_numpy(synth.quantize(synth.smooth_noise_np(321, 481, 6),
                                         4)).cuda(), 32),
        (torch.from_numpy(rng.integers(0, 3, size=(300, 517))
                          .astype(np.uint8)).cuda(), 16),
        (torch.from_numpy(synth.checkerboard(700, 900, 3)).cuda(), 64),
    ]


def test_static_scratch_matches_workspace_entry_point():
    pkg = package()
    lib = pkg.lib()
    for image, tile in cases():
        want_max, want_min = pkg.extrema(image, tile=tile, check=True)
        for call in range(2):
            mx = torch.full_like(image, 7)
            mn = torch.full_like(image, 7)
            assert call_static(lib, image, tile, mx, mn) == 0
            rc, stats = read_static_status(pkg, lib)
            assert rc == 0 and stats.device_error == 0, (rc, tile, call)
            assert stats.tiles == ((image.shape[0] + tile - 1) // tile) * \
                ((image.shape[1] + tile - 1) // tile)
            assert torch.equal(mx, want_max), (image.shape, tile, call)
            assert torch.equal(mn, want_min), (image.shape, tile, call)


def test_static_scratch_allocates_nothing_after_warm_up():
    pkg = package()
    lib = pkg.lib()
    work = cases()
    outs = [(torch.empty_like(im), torch.empty_like(im)) for im, _ in work]
    # Warm-up: loads the module holding the array and sets it up.
    for (image, tile), (mx, mn) in zip(work, outs):
        assert call_static(lib, image, tile, mx, mn) == 0
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    allocs_before = torch.cuda.memory_stats().get("allocation.all.allocated",
                                                  0)
    for _ in range(3):
        for (image, tile), (mx, mn) in zip(work, outs):
            assert call_static(lib, image, tile, mx, mn) == 0
    torch.cuda.synchronize()
    assert read_static_status(pkg, lib)[0] == 0
    free_after, _ = torch.cuda.mem_get_info()
    allocs_after = torch.cuda.memory_stats().get("allocation.all.allocated", 0)
    assert free_after == free_before
    assert allocs_after == allocs_before


FRESH = r"""
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, {root!r})
import importlib
pkg = importlib.import_module("sparse-seam_b200")
lib = pkg.lib()
stats = pkg.Stats()
s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
# Nothing set up yet in this process's context.
assert lib.ss_static_scratch_read_status(s, ctypes.byref(stats)) == 11
rng = np.random.default_rng(3)
img = torch.from_numpy((rng.integers(0, 256, size=(777, 1029)) >> 5 << 5)
                       .astype(np.uint8)).cuda()
want = pkg.extrema(img, tile=32, check=True)
for call in range(2):
    mx = torch.full_like(img, 7)
    mn = torch.full_like(img, 7)
    rc = lib.ss_extrema_static_scratch(img.data_ptr(), 1029, 777, 1029, 32,
                                       mx.data_ptr(), mn.data_ptr(), 1029, s)
    assert rc == 0, rc
    assert lib.ss_static_scratch_read_status(s, ctypes.byref(stats)) == 0
    assert torch.equal(mx, want[0]) and torch.equal(mn, want[1]), call
print("OK")
"""


def test_static_scratch_first_call_in_a_fresh_process():
    out = subprocess.run([sys.executable, "-c", FRESH.format(root=ROOT)],
                         capture_output=True, text=True, timeout=600,
                         cwd=ROOT, env=dict(os.environ))
    assert out.returncode == 0 and out.stdout.strip().endswith("OK"), \
        out.stdout + out.stderr


def test_static_scratch_refuses_images_beyond_its_capacity():
    pkg = package()
    lib = pkg.lib()
    image = torch.zeros((4096, 4096), dtype=torch.uint8, device="cuda")
    mx = torch.full_like(image, 7)
    mn = torch.full_like(image, 7)
    assert call_static(lib, image, 32, mx, mn) == 13
    torch.cuda.synchronize()
    assert int(mx.max()) == 7 and int(mx.min()) == 7
