"""Image files: the library's PGM / PNG reader gives the bytes the reference's
reader (OpenCV, cv::imread(path, IMREAD_GRAYSCALE)) gives.  PNGs of every
colour type, bit depth and scanline filter are written here with zlib; the
comparison runs where OpenCV's Python module is installed."""
import struct
import zlib

import numpy as np
import pytest

from conftest import package


def _chunk(kind: bytes, body: bytes) -> bytes:
    return (struct.pack(">I", len(body)) + kind + body +
            struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF))


def _filter_row(raw: bytes, prev: bytes, bpp: int, ftype: int) -> bytes:
    out = bytearray(raw)
    for i in range(len(raw)):
        a = raw[i - bpp] if i >= bpp else 0
        b = prev[i]
        c = prev[i - bpp] if i >= bpp else 0
        if ftype == 1:
            pred = a
        elif ftype == 2:
            pred = b
        elif ftype == 3:
            pred = (a + b) >> 1
        elif ftype == 4:
            p = a + b - c
            pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
            pred = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
        else:
            pred = 0
        out[i] = (raw[i] - pred) & 0xFF
    return bytes([ftype]) + bytes(out)


def write_png(path, rows: np.ndarray, ctype: int, depth: int, palette=None,
              seed: int = 0):
    """rows: (h, row_bytes) uint8 of packed samples."""
    h = rows.shape[0]
    channels = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
    width = rows.shape[1] * 8 // (channels * depth)
    bpp = max(1, channels * depth // 8)
    rng = np.random.default_rng(seed)
    data = bytearray()
    prev = bytes(rows.shape[1])
    for y in range(h):
        raw = rows[y].tobytes()
        data += _filter_row(raw, prev, bpp, int(rng.integers(0, 5)))
        prev = raw
    png = b"\x89PNG\r\n\x1a\n"
    png += _chunk(b"IHDR", struct.pack(">IIBBBBB", width, h, depth, ctype,
                                       0, 0, 0))
    if palette is not None:
        png += _chunk(b"PLTE", palette.astype(np.uint8).tobytes())
    comp = zlib.compress(bytes(data), 6)
    # Several IDAT chunks.
    for k in range(0, len(comp), 97):
        png += _chunk(b"IDAT", comp[k:k + 97])
    png += _chunk(b"IEND", b"")
    with open(path, "wb") as f:
        f.write(png)
    return width


CASES = [(0, 8), (0, 1), (0, 2), (0, 4), (2, 8), (3, 8), (3, 4), (3, 1),
         (4, 8), (6, 8)]


@pytest.mark.parametrize("ctype,depth", CASES)
def test_png_matches_opencv(tmp_path, ctype, depth):
    cv2 = pytest.importorskip("cv2")
    pkg = package()
    rng = np.random.default_rng(ctype * 16 + depth)
    for trial, (h, w) in enumerate([(1, 1), (7, 13), (33, 50), (64, 3)]):
        channels = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
        row_bytes = (w * channels * depth + 7) // 8
        palette = None
        if ctype == 3:
            colors = 1 << depth
            palette = rng.integers(0, 256, size=(colors, 3))
        rows = rng.integers(0, 256, size=(h, row_bytes)).astype(np.uint8)
        if depth < 8:
            # Zero the padding bits after the last sample of each row.
            used = w * channels * depth
            if used % 8:
                rows[:, -1] &= (0xFF << (8 - used % 8)) & 0xFF
        path = str(tmp_path / f"c{ctype}d{depth}_{trial}.png")
        assert write_png(path, rows, ctype, depth, palette, seed=trial) >= w
        want = cv2.imread(path, cv2.IMREAD_GRAYSCALE)
        assert want is not None
        got = pkg.read_image(path)
        assert got.shape == want.shape[:2], (ctype, depth, trial)
        assert np.array_equal(got, want), (ctype, depth, trial,
                                           int((got != want).sum()))


def test_pgm_round_trip_and_opencv(tmp_path):
    pkg = package()
    rng = np.random.default_rng(1)
    img = rng.integers(0, 256, size=(37, 53)).astype(np.uint8)
    path = str(tmp_path / "a.pgm")
    pkg.write_pgm(path, img)
    assert np.array_equal(pkg.read_image(path), img)
    # ASCII PGM with comments and a maxval below 255.
    p2 = tmp_path / "b.pgm"
    small = rng.integers(0, 16, size=(4, 5))
    p2.write_text("P2\n# comment\n5 4\n# another\n15\n" +
                  "\n".join(" ".join(str(v) for v in r) for r in small) + "\n")
    got = pkg.read_image(str(p2))
    assert got.shape == (4, 5)
    try:
        import cv2
    except ImportError:
        return
    assert np.array_equal(pkg.read_image(path),
                          cv2.imread(path, cv2.IMREAD_GRAYSCALE))
    assert np.array_equal(got, cv2.imread(str(p2), cv2.IMREAD_GRAYSCALE))


def test_bad_files_are_refused(tmp_path):
    pkg = package()
    bad = tmp_path / "x.pgm"
    bad.write_bytes(b"P5\n3 3\n255\n\x00\x01")   # truncated
    with pytest.raises(pkg.SparseSeamError):
        pkg.read_image(str(bad))
    with pytest.raises(pkg.SparseSeamError):
        pkg.read_image(str(tmp_path / "missing.png"))
    notimg = tmp_path / "y.png"
    notimg.write_bytes(b"\x89PNG\r\n\x1a\n" + b"\x00" * 20)
    with pytest.raises(pkg.SparseSeamError):
        pkg.read_image(str(notimg))
