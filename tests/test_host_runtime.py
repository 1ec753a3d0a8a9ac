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
                    max_batch_images=16, reserved=0, batch_tiles=1000,
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
    table = at.TuningTable({k: cands[k] for k in range(4)},
                           {0: {"x": 1.0}})
    back = at.TuningTable.from_json(table.to_json())
    assert back.choices == table.choices
    assert back.choice_for(700, 700) == cands[3]
