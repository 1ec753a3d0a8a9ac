"""The C ABI library loads, exports every declared symbol, and validates its
arguments on the host (no GPU needed: nothing here reaches a CUDA call)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, package

HEADER = os.path.join(ROOT, "include", "sparse_seam.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(ss_[a-z_0-9]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    pkg = package()
    lib = pkg.lib()
    names = declared_functions()
    assert names == sorted(pkg.SIGNATURES), "header and bindings disagree"
    for name in names:
        assert hasattr(lib, name), name
        assert name in pkg.SIGNATURES, f"{name} has no ctypes signature"


def test_status_strings_and_version():
    pkg = package()
    lib = pkg.lib()
    assert lib.ss_abi_version() == 2
    for code, name in pkg.STATUS.items():
        assert lib.ss_status_string(code).decode() == name
    assert lib.ss_status_string(999).decode() == "SS_ERR_UNKNOWN"


def test_workspace_bytes():
    pkg = package()
    # Sizes grow with the image and shrink with the tile edge.
    a = pkg.workspace_bytes(512, 512, 32)
    b = pkg.workspace_bytes(1024, 1024, 32)
    c = pkg.workspace_bytes(1024, 1024, 64)
    assert a % 256 == 0 and b > a and c < b
    # 2040x1356 at T=32: 64 x 43 tiles, 128 slots of 9 bytes each, border
    # records, counters, a run log of up to 32 x 32 entries of 4 bytes and
    # up to 384 seam items of 4 bytes per tile -> about 7 bytes per pixel.
    w = pkg.workspace_bytes(2040, 1356, 32)
    assert 2752 * (128 * 9 + 4096 + 1536) < w < 2040 * 1356 * 7.5
    # T=64 (row-scan kernels, 64 x 64 tiles): 32 x 22 tiles, 256 slots of 9
    # bytes, a run log of up to 64 x 64 entries and 768 seam items per tile
    # -> about 5.3 bytes per pixel.
    w64 = pkg.workspace_bytes(2040, 1356, 64)
    assert 704 * (256 * 9 + 16384 + 3072) < w64 < 2040 * 1356 * 6
    with pytest.raises(pkg.SparseSeamError) as e:
        pkg.workspace_bytes(100, 100, 48)
    assert e.value.status == 2
    with pytest.raises(pkg.SparseSeamError) as e:
        pkg.workspace_bytes(0, 100, 32)
    assert e.value.status == 1
    with pytest.raises(pkg.SparseSeamError) as e:
        pkg.workspace_bytes(200000, 200000, 16)
    assert e.value.status == 5


def test_extrema_rejects_bad_arguments_before_any_cuda_call():
    lib = package().lib()
    ws = 256 * 1000
    fake = 0x10000  # never dereferenced: validation fails first
    # NULL image
    assert lib.ss_extrema(None, 10, 10, 10, 32, fake, fake, 10, fake, ws,
                          None) == 1
    # pitch < width
    assert lib.ss_extrema(fake, 10, 10, 9, 32, fake, fake, 10, fake, ws,
                          None) == 1
    # out_pitch < width
    assert lib.ss_extrema(fake, 10, 10, 10, 32, fake, fake, 9, fake, ws,
                          None) == 1
    # unsupported tile
    assert lib.ss_extrema(fake, 10, 10, 10, 24, fake, fake, 10, fake, ws,
                          None) == 2
    # misaligned workspace
    assert lib.ss_extrema(fake, 10, 10, 10, 32, fake, fake, 10, fake + 8, ws,
                          None) == 4
    # workspace too small
    assert lib.ss_extrema(fake, 1000, 1000, 1000, 32, fake, fake, 1000, fake,
                          4096, None) == 3
    assert lib.ss_workspace_init(fake + 8, 4096, None) == 4
    assert lib.ss_workspace_init(None, 4096, None) == 1


def test_batch_plan_is_built_on_the_host():
    pkg = package()
    lib = pkg.lib()
    sizes = [(5, 7), (64, 64), (33, 100), (1, 1)]
    descs = (pkg.ImageDesc * len(sizes))()
    for i, (h, w) in enumerate(sizes):
        base = 0x1000000 * (i + 1)
        descs[i] = pkg.ImageDesc(base, base + 0x100000, base + 0x200000,
                                 w, h, w + 3, w)
    tiles = ctypes.c_int64()
    assert lib.ss_batch_tiles(descs, len(sizes), 32, ctypes.byref(tiles)) == 0
    want = sum(-(-w // 32) * -(-h // 32) for h, w in sizes)
    assert tiles.value == want
    nbytes = ctypes.c_size_t()
    assert lib.ss_batch_plan_bytes(len(sizes), tiles.value,
                                   ctypes.byref(nbytes)) == 0
    plan = np.zeros(nbytes.value, dtype=np.uint8)
    ws = ctypes.c_size_t()
    assert lib.ss_batch_plan_fill(descs, len(sizes), 32, plan.ctypes.data,
                                  nbytes.value, ctypes.byref(ws)) == 0
    # Header: magic, count, tile, total tiles.
    head = plan[:64].view(np.int32)
    assert head[1] == len(sizes) and head[2] == 32
    assert plan[16:24].view(np.int64)[0] == want
    # Image table: 64-byte entries; tile_base is the running tile sum.
    table = plan[64:64 + 64 * len(sizes)].reshape(len(sizes), 64)
    bases = [int(row[48:56].view(np.int64)[0]) for row in table]
    expect = np.cumsum([0] + [-(-w // 32) * -(-h // 32)
                              for h, w in sizes])[:-1].tolist()
    assert bases == expect
    for row, (h, w) in zip(table, sizes):
        dims = row[24:48].view(np.int32)
        assert dims[0] == w and dims[1] == h and dims[2] == w + 3
        assert dims[4] == -(-w // 32) and dims[5] == -(-h // 32)
    # Tile -> image map.
    off = 64 + 64 * len(sizes)
    tmap = plan[off:off + 4 * want].view(np.int32).tolist()
    expect_map = []
    for i, (h, w) in enumerate(sizes):
        expect_map += [i] * (-(-w // 32) * -(-h // 32))
    assert tmap == expect_map
    assert ws.value == pkg.workspace_bytes(1, 1, 32) or ws.value > 0
    # A bad descriptor is rejected.
    descs[2].pitch = 1
    assert lib.ss_batch_tiles(descs, len(sizes), 32, ctypes.byref(tiles)) == 1


def test_kernel_config_hook():
    pkg = package()
    for tile, choices in pkg.KERNEL_CONFIGS.items():
        default = pkg.get_kernel_config(tile)
        assert default in choices
        for w in choices:
            pkg.set_kernel_config(tile, w)
            assert pkg.get_kernel_config(tile) == w
        pkg.set_kernel_config(tile, default)
    with pytest.raises(pkg.SparseSeamError) as e:
        pkg.set_kernel_config(32, 3)
    assert e.value.status == 1
    with pytest.raises(pkg.SparseSeamError) as e:
        pkg.set_kernel_config(64, -2)
    assert e.value.status == 1


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    pkg = package()
    monkeypatch.setattr(pkg, "_LIB", None)
    monkeypatch.setattr(pkg, "LIBRARY", str(tmp_path / "absent.so"))
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        pkg.lib()
