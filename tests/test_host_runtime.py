"""Host-side runtime pieces that need no GPU: the serving pool allocator,
the serving loop's argument checks, the batch-launch checks and the
autotuner's bookkeeping."""
import ctypes
import importlib
import os
import shutil
import subprocess

import pytest

from conftest import ROOT, package

CSRC = os.path.join(ROOT, "sparse-seam_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_pool_allocator_randomised(tmp_path):
    exe = str(tmp_path / "pool_check")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I" + CSRC, "-o", exe,
                           os.path.join(ROOT, "tests", "native",
                                        "pool_check.cpp")])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "OK", out.stdout


def test_server_config_is_checked_before_any_cuda_call():
    pkg = package()
    lib = pkg.lib()
    h = ctypes.c_void_p()

    def create(**kw):
        base = dict(device=0, tile=32, persistent=1, inflight=2,
                    max_batch_images=16, unpack_threads=0, batch_tiles=1000,
                    pool_bytes=1 << 20)
        base.update(kw)
        cfg = pkg.ServerConfig(**base)
        return lib.ss_server_create(ctypes.byref(cfg), ctypes.byref(h))

    assert create(tile=48) == 2
    assert create(inflight=0) == 1
    assert create(inflight=17) == 1
    assert create(max_batch_images=0) == 1
    assert create(batch_tiles=0) == 1
    assert create(device=-1) == 1
    assert create(batch_tiles=1 << 40) == 5
    assert create(unpack_threads=-2) == 1
    assert lib.ss_server_create(None, ctypes.byref(h)) == 1
    # Calls on a null server are refused, never dereferenced.
    req = pkg.Request()
    assert lib.ss_server_submit(None, ctypes.byref(req), None) == 1
    n = ctypes.c_int()
    buf = (pkg.Completion * 4)()
    assert lib.ss_server_poll(None, buf, 4, ctypes.byref(n), 0) == 1
    st = pkg.ServerStats()
    assert lib.ss_server_get_stats(None, ctypes.byref(st)) == 1
    lib.ss_server_destroy(None)


def test_batch_launch_rejects_bad_choices():
    pkg = package()
    lib = pkg.lib()
    fake = 0x10000   # never dereferenced: validation fails first
    bad_group = pkg.Launch(0, 0, 3, 0)
    assert lib.ss_extrema_batch_launch(fake, fake, 4096,
                                       ctypes.byref(bad_group), fake, 4096,
                                       None) == 1
    bad_passes = pkg.Launch(0, 0, 0, 9)
    assert lib.ss_extrema_batch_launch(fake, fake, 4096,
                                       ctypes.byref(bad_passes), fake, 4096,
                                       None) == 1
    bad_flatten = pkg.Launch(0, 0, 0, 0, 3)
    assert lib.ss_extrema_batch_launch(fake, fake, 4096,
                                       ctypes.byref(bad_flatten), fake, 4096,
                                       None) == 1
    assert lib.ss_extrema_batch_launch(None, fake, 4096, None, fake, 4096,
                                       None) == 1


def test_autotuner_tables():
    at = importlib.import_module("sparse-seam_b200.autotune")
    pkg = package()
    # Classes partition the areas.
    assert at.size_class(1, 1) == 0
    assert at.size_class(127, 128) == 0
    assert at.size_class(128, 128) == 1
    assert at.size_class(256, 256) == 2
    assert at.size_class(512, 512) == 3
    assert at.size_class(8192, 8192) == 3
    cands = at.candidates()
    assert cands[0].tile == 32 and cands[0].warps == pkg.get_kernel_config(32)
    assert len(set(cands)) == len(cands)
    for tile, family in pkg.KERNEL_CONFIGS.items():
        for w in family:
            assert any(c.tile == tile and c.warps == w for c in cands)
    assert {c.flatten for c in cands if c.warps < 0} == {0, 1, 2}
    table = at.TuningTable({k: cands[k] for k in range(4)},
                           {0: {"x": 1.0}}, cands[5], {"y": 2.0})
    back = at.TuningTable.from_json(table.to_json())
    assert back.choices == table.choices
    assert back.mix == cands[5] and back.mix_timings_ms == {"y": 2.0}
    assert back.choice_for(700, 700) == cands[3]


def test_unpack_masks_on_the_host():
    """The host half of the compact transfer: bit planes (bit i of word
    i / 32 for pixel i) back to 0/255 bytes, any length, any thread count."""
    import numpy as np
    pkg = package()
    lib = pkg.lib()
    rng = np.random.default_rng(4)
    for n in (0, 1, 7, 15, 16, 17, 31, 32, 33, 47, 1000, 65536,
              65536 * 3 + 17, 65536 * 2 + 31):
        want_max = (rng.random(n) < 0.3).astype(np.uint8) * 255
        want_min = (rng.random(n) < 0.6).astype(np.uint8) * 255
        words = (n + 31) // 32
        bmax = np.zeros(words * 4, np.uint8)
        bmin = np.zeros(words * 4, np.uint8)
        pm = np.packbits(want_max != 0, bitorder="little")
        pn = np.packbits(want_min != 0, bitorder="little")
        bmax[:pm.size] = pm
        bmin[:pn.size] = pn
        for threads, shift in ((1, 0), (3, 5), (0, 13), (2, 1)):
            # Outputs at every alignment: the streaming middle and the
            # byte-wise head and tail must join up.
            buf_max = np.full(n + 40, 9, np.uint8)
            buf_min = np.full(n + 40, 9, np.uint8)
            out_max = buf_max[shift:shift + n + 5]
            out_min = buf_min[shift:shift + n + 5]
            assert lib.ss_unpack_masks(bmax.ctypes.data, bmin.ctypes.data, n,
                                       out_max.ctypes.data,
                                       out_min.ctypes.data, threads) == 0
            assert np.array_equal(out_max[:n], want_max), (n, threads, shift)
            assert np.array_equal(out_min[:n], want_min), (n, threads, shift)
            assert (out_max[n:] == 9).all() and (out_min[n:] == 9).all()
            assert (buf_max[:shift] == 9).all()
    assert lib.ss_unpack_masks(None, None, 4, None, None, 1) == 1


@pytest.mark.parametrize("simd", ["0", "1", "2"])
def test_unpack_masks_every_simd_path(simd):
    """The scalar, AVX2 and AVX-512 expansions (as far as this CPU has them)
    agree with numpy, run in a child process with the level capped."""
    import sys
    code = (
        "import sys; sys.path.insert(0, %r); sys.path.insert(0, %r)\n"
        "import test_host_runtime as t\n"
        "t.test_unpack_masks_on_the_host()\n"
        "print('OK')\n" % (ROOT, os.path.join(ROOT, "tests")))
    env = dict(os.environ, SS_UNPACK_SIMD=simd)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True,
                         text=True, timeout=300, env=env, cwd=ROOT)
    assert out.returncode == 0 and "OK" in out.stdout, out.stderr[-2000:]
