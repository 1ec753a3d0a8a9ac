"""The zero-allocation entry point against the workspace entry point.

ss_extrema_static_scratch serves callers that cannot allocate device memory:
its scratch is a fixed array inside the library.  Its masks must equal those
of ss_extrema (bytes, so exactly) on two calls in a row, from a fresh process
(the first call sets the array up) as well as after other tests; images
beyond the array's capacity are refused without touching the outputs.
"""
import ctypes

import numpy as np
import pytest

from conftest import package

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def call_static(lib, image, tile, maxima, minima):
    h, w = image.shape
    stream = torch.cuda.current_stream().cuda_stream
    return lib.ss_extrema_static_scratch(
        image.data_ptr(), w, h, image.stride(0), tile, maxima.data_ptr(),
        minima.data_ptr(), maxima.stride(0), ctypes.c_void_p(stream))


def test_static_scratch_matches_workspace_entry_point():
    import importlib
    pkg = package()
    lib = pkg.lib()
    synth = importlib.import_module("sparse-seam_b200.synth")
    rng = np.random.default_rng(17)
    cases = [
        (synth.smooth_noise(1356, 2040, seed=5, device="cuda"), 32),
        (torch.from_numpy(synth.quantize(synth.smooth_noise_np(321, 481, 6),
                                         4)).cuda(), 32),
        (torch.from_numpy(rng.integers(0, 3, size=(300, 517))
                          .astype(np.uint8)).cuda(), 16),
        (torch.from_numpy(synth.checkerboard(700, 900, 3)).cuda(), 64),
    ]
    for image, tile in cases:
        want_max, want_min = pkg.extrema(image, tile=tile, check=True)
        for call in range(2):
            mx = torch.full_like(image, 7)
            mn = torch.full_like(image, 7)
            assert call_static(lib, image, tile, mx, mn) == 0
            torch.cuda.synchronize()
            assert torch.equal(mx, want_max), (image.shape, tile, call)
            assert torch.equal(mn, want_min), (image.shape, tile, call)


def test_static_scratch_refuses_images_beyond_its_capacity():
    pkg = package()
    lib = pkg.lib()
    image = torch.zeros((4096, 4096), dtype=torch.uint8, device="cuda")
    mx = torch.full_like(image, 7)
    mn = torch.full_like(image, 7)
    assert call_static(lib, image, 32, mx, mn) == 13
    torch.cuda.synchronize()
    assert int(mx.max()) == 7 and int(mx.min()) == 7
