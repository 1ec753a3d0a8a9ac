"""Host-to-host forms on the GPU: the compact (bit-plane) read-back and the
byte read-back give the oracle's masks."""
import importlib

import numpy as np
import pytest

import oracle
from conftest import package

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_pack_masks_matches_numpy():
    pkg = package()
    lib = pkg.lib()
    rng = np.random.default_rng(2)
    for n in (1, 31, 32, 33, 255, 256, 257, 100_000, 1_000_003):
        mx = torch.from_numpy((rng.random(n) < 0.4).astype(np.uint8) * 255)
        mn = torch.from_numpy((rng.random(n) < 0.7).astype(np.uint8) * 255)
        words = (n + 31) // 32
        d_bits = torch.full((2, words + 1), -1, dtype=torch.int32,
                            device="cuda")
        assert lib.ss_pack_masks(mx.cuda().data_ptr(), mn.cuda().data_ptr(),
                                 n, d_bits[0].data_ptr(),
                                 d_bits[1].data_ptr(), None) == 0
        torch.cuda.synchronize()
        bits = d_bits.cpu().numpy().view(np.uint8).reshape(2, -1)
        for plane, m in ((0, mx), (1, mn)):
            want = np.packbits(m.numpy() != 0, bitorder="little")
            got = bits[plane][:want.size]
            assert np.array_equal(got, want), (n, plane)
            # The word after the last is untouched.
            assert (bits[plane][words * 4:] == 0xFF).all()


@pytest.mark.parametrize("packed", [True, False])
def test_host_batch_matches_oracle(packed):
    host = importlib.import_module("sparse-seam_b200.host")
    synth = importlib.import_module("sparse-seam_b200.synth")
    images = [t.cpu().numpy() for t in
              synth.uneven_batch(37, seed=31, lo=9, hi=700)]
    hb = host.HostBatch(images, tile=32, chunks=5, packed=packed)
    for rep in range(2):
        for m in hb.maxima + hb.minima:
            m[...] = 7
        end = hb.run()
        end.synchronize()
        hb.check()
        for i, im in enumerate(images):
            want = oracle.extrema(im)
            assert np.array_equal(hb.maxima[i], want[0]), (packed, rep, i)
            assert np.array_equal(hb.minima[i], want[1]), (packed, rep, i)
    if packed:
        assert hb.d2h_bytes < hb.pixels // 3


def test_host_batch_thread_tuning_keeps_masks():
    """tune_threads picks one of the candidates by timing; passes at the
    picked count still give the oracle's masks."""
    host = importlib.import_module("sparse-seam_b200.host")
    synth = importlib.import_module("sparse-seam_b200.synth")
    images = [t.cpu().numpy() for t in
              synth.uneven_batch(12, seed=5, lo=40, hi=500)]
    hb = host.HostBatch(images, tile=32, chunks=3, packed=True)
    picked = hb.tune_threads(candidates=(1, 2, 3), reps=1)
    assert picked in (1, 2, 3) and hb.threads == picked
    for m in hb.maxima + hb.minima:
        m[...] = 7
    hb.run().synchronize()
    hb.check()
    for i, im in enumerate(images):
        want = oracle.extrema(im)
        assert np.array_equal(hb.maxima[i], want[0]), i
        assert np.array_equal(hb.minima[i], want[1]), i
