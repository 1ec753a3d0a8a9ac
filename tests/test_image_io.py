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


# ---- BMP --------------------------------------------------------------------

def write_bmp(path, pixel_rows, width, height, bpp, comp=0, palette=None,
              masks=None, top_down=False, header=40, stream=None):
    """A BMP file: `pixel_rows` top row first (packed bytes per row), or an
    RLE `stream` (comp 1 / 2).  header 12 = OS/2 core, 40 = info (+ bit-field
    masks after it), 108 / 124 = V4 / V5 (masks inside)."""
    if stream is None:
        stride = (width * bpp + 31) // 32 * 4
        order = pixel_rows if top_down else pixel_rows[::-1]
        data = b"".join(bytes(r) + b"\0" * (stride - len(r)) for r in order)
    else:
        data = stream
    pal = b""
    if palette is not None:
        entry = 3 if header == 12 else 4
        pal = b"".join(bytes([c[2], c[1], c[0], 0][:entry]) for c in palette)
    if header == 12:
        dib = struct.pack("<IHHHH", 12, width, height, 1, bpp)
        extra = b""
    else:
        dib = struct.pack("<IiiHHIIiiII", header, width,
                          -height if top_down else height, 1, bpp, comp,
                          len(data), 2835, 2835,
                          0 if palette is None else len(palette), 0)
        extra = b""
        if masks is not None and header == 40:
            extra = struct.pack("<III", *masks)
        if header > 40:
            m = masks or (0, 0, 0)
            dib += struct.pack("<IIII", m[0], m[1], m[2], 0)
            dib += b"\0" * (header - 56)
    off = 14 + len(dib) + len(extra) + len(pal)
    with open(path, "wb") as f:
        f.write(b"BM" + struct.pack("<IHHI", off + len(data), 0, 0, off) +
                dib + extra + pal + data)


def rle_stream(rng, width, height, rle4):
    """A well-formed RLE8 / RLE4 stream with encoded runs, literal runs,
    in-row moves, short rows and an end-of-bitmap mark."""
    colors = 16 if rle4 else 256
    out = bytearray()
    for _ in range(height):
        x = 0
        stop = width if rng.random() < 0.8 else int(rng.integers(0, width + 1))
        while x < stop:
            left = stop - x
            kind = rng.random()
            if kind < 0.45 or left < 3:
                n = int(rng.integers(1, min(255, left) + 1))
                a, b = rng.integers(0, colors, size=2)
                out += bytes([n, (a << 4 | b) if rle4 else a])
            elif kind < 0.9:
                n = int(rng.integers(3, min(255, left) + 1))
                idx = rng.integers(0, colors, size=n)
                if rle4:
                    idx = np.concatenate([idx, [0]]) if n % 2 else idx
                    lit = bytes(int(idx[i] << 4 | idx[i + 1])
                                for i in range(0, len(idx), 2))
                else:
                    lit = bytes(int(v) for v in idx)
                if len(lit) % 2:
                    lit += b"\0"
                out += bytes([0, n]) + lit
            elif left > 1:
                # A move stays inside the row (OpenCV 4.13 skips one more row
                # after a move that ends exactly at the row's end).
                dx = int(rng.integers(1, min(255, left - 1) + 1))
                out += bytes([0, 2, dx, 0])
                n = dx
            else:
                continue
            x += n
        out += bytes([0, 0])
    out += bytes([0, 1])
    # Bytes after the end mark are ignored; OpenCV's buffered reader wants a
    # few there.
    return bytes(out) + bytes(32)


def test_bmp_matches_opencv(tmp_path):
    cv2 = pytest.importorskip("cv2")
    pkg = package()
    rng = np.random.default_rng(7)
    cases = []
    for (h, w) in [(1, 1), (7, 13), (33, 50), (64, 3)]:
        start = len(cases)
        for bpp in (1, 4, 8):
            ncol = int(rng.integers(2, (1 << bpp) + 1))
            pal = rng.integers(0, 256, size=(ncol, 3))
            idx = rng.integers(0, ncol, size=(h, w))
            rows = []
            for y in range(h):
                bits = "".join(format(int(v), f"0{bpp}b") for v in idx[y])
                bits += "0" * (-len(bits) % 8)
                rows.append(bytes(int(bits[i:i + 8], 2)
                                  for i in range(0, len(bits), 8)))
            cases.append(dict(pixel_rows=rows, bpp=bpp, palette=pal))
            # A core header's palette always has 2^bpp entries.
            full = np.concatenate(
                [pal, rng.integers(0, 256, size=((1 << bpp) - ncol, 3))])
            cases.append(dict(pixel_rows=rows, bpp=bpp,
                              palette=full if bpp == 8 else pal,
                              header=12 if bpp == 8 else 40,
                              top_down=bpp == 4))
        v16 = rng.integers(0, 65536, size=(h, w)).astype("<u2")
        r16 = [v16[y].tobytes() for y in range(h)]
        cases.append(dict(pixel_rows=r16, bpp=16))
        cases.append(dict(pixel_rows=r16, bpp=16, comp=3,
                          masks=(0xF800, 0x07E0, 0x001F)))
        cases.append(dict(pixel_rows=r16, bpp=16, comp=3,
                          masks=(0x7C00, 0x03E0, 0x001F)))
        c3 = rng.integers(0, 256, size=(h, w, 3)).astype(np.uint8)
        r24 = [c3[y].tobytes() for y in range(h)]
        cases.append(dict(pixel_rows=r24, bpp=24))
        cases.append(dict(pixel_rows=r24, bpp=24, top_down=True))
        cases.append(dict(pixel_rows=r24, bpp=24, header=12))
        c4 = rng.integers(0, 256, size=(h, w, 4)).astype(np.uint8)
        r32 = [c4[y].tobytes() for y in range(h)]
        cases.append(dict(pixel_rows=r32, bpp=32))
        cases.append(dict(pixel_rows=r32, bpp=32, comp=3, header=124,
                          masks=(0x00FF0000, 0x0000FF00, 0x000000FF)))
        for rle4 in (False, True):
            ncol = 16 if rle4 else 256
            pal = rng.integers(0, 256, size=(ncol, 3))
            cases.append(dict(pixel_rows=None, bpp=4 if rle4 else 8,
                              comp=2 if rle4 else 1, palette=pal,
                              stream=rle_stream(rng, w, h, rle4)))
        for c in cases[start:]:
            c["size"] = (w, h)
    for k, c in enumerate(cases):
        w, h = c.pop("size")
        path = str(tmp_path / f"b{k}.bmp")
        write_bmp(path, c.pop("pixel_rows"), w, h, **c)
        want = cv2.imread(path, cv2.IMREAD_GRAYSCALE)
        assert want is not None, (k, c.get("bpp"), c.get("comp"))
        got = pkg.read_image(path)
        assert got.shape == want.shape, k
        assert np.array_equal(got, want), (k, c.get("bpp"), c.get("comp"),
                                           int((got != want).sum()))


def test_bad_bmp_files_are_refused(tmp_path):
    pkg = package()
    good = tmp_path / "g.bmp"
    rows = [bytes([1, 2, 3]) * 4 for _ in range(4)]
    write_bmp(str(good), rows, 4, 4, 24)
    data = good.read_bytes()
    assert pkg.read_image(str(good)).shape == (4, 4)
    cut = tmp_path / "cut.bmp"
    cut.write_bytes(data[:-10])                  # rows missing
    bad_bpp = tmp_path / "bpp.bmp"
    bad_bpp.write_bytes(data[:28] + struct.pack("<H", 7) + data[30:])
    bad_comp = tmp_path / "comp.bmp"
    bad_comp.write_bytes(data[:30] + struct.pack("<I", 9) + data[34:])
    run = tmp_path / "run.bmp"                  # an RLE8 run past the row
    write_bmp(str(run), None, 4, 1, 8, comp=1, palette=[(0, 0, 0)] * 2,
              stream=bytes([9, 1, 0, 1]))
    for f in (cut, bad_bpp, bad_comp, run):
        with pytest.raises(pkg.SparseSeamError):
            pkg.read_image(str(f))


def test_bmp_v4_bit_fields(tmp_path):
    """16-bit bit fields inside a V4 / V5 header (which OpenCV 4.13 refuses)
    decode as the same pixels with the fields after a 40-byte header."""
    pkg = package()
    rng = np.random.default_rng(9)
    v = rng.integers(0, 65536, size=(9, 11)).astype("<u2")
    rows = [v[y].tobytes() for y in range(9)]
    for masks in ((0x7C00, 0x03E0, 0x001F), (0xF800, 0x07E0, 0x001F)):
        outs = []
        for header in (40, 108, 124):
            path = str(tmp_path / f"v{header}.bmp")
            write_bmp(path, rows, 11, 9, 16, comp=3, masks=masks,
                      header=header)
            outs.append(pkg.read_image(path))
        assert all(np.array_equal(outs[0], o) for o in outs[1:])


# ---- JPEG -------------------------------------------------------------------

JPEG_PARAMS = [
    ("q95", "IMWRITE_JPEG_QUALITY", 95),
    ("q20", "IMWRITE_JPEG_QUALITY", 20),
    ("q100", "IMWRITE_JPEG_QUALITY", 100),
    ("444", "IMWRITE_JPEG_SAMPLING_FACTOR", "IMWRITE_JPEG_SAMPLING_FACTOR_444"),
    ("422", "IMWRITE_JPEG_SAMPLING_FACTOR", "IMWRITE_JPEG_SAMPLING_FACTOR_422"),
    ("411", "IMWRITE_JPEG_SAMPLING_FACTOR", "IMWRITE_JPEG_SAMPLING_FACTOR_411"),
    ("restart3", "IMWRITE_JPEG_RST_INTERVAL", 3),
    ("optimised", "IMWRITE_JPEG_OPTIMIZE", 1),
    ("progressive", "IMWRITE_JPEG_PROGRESSIVE", 1),
]


def _jpeg_inputs(rng):
    for (h, w) in [(1, 1), (7, 13), (33, 50), (64, 3), (17, 16), (321, 481)]:
        noise = rng.integers(0, 256, size=(h, w, 3)).astype(np.uint8)
        yy, xx = np.mgrid[0:h, 0:w]
        smooth = np.stack([(xx * 5 + yy * 3) % 256, (xx * 2 + yy * 7) % 256,
                           (xx * 11) % 256], -1).astype(np.uint8)
        yield noise
        yield smooth
        yield noise[..., 0].copy()   # one-component file


@pytest.mark.parametrize("name,key,value", JPEG_PARAMS,
                         ids=[p[0] for p in JPEG_PARAMS])
def test_jpeg_matches_opencv(tmp_path, name, key, value):
    cv2 = pytest.importorskip("cv2")
    pkg = package()
    rng = np.random.default_rng(11)
    if isinstance(value, str):
        value = getattr(cv2, value)
    for k, img in enumerate(_jpeg_inputs(rng)):
        ok, buf = cv2.imencode(".jpg", img, [getattr(cv2, key), value])
        assert ok
        path = str(tmp_path / f"{name}_{k}.jpg")
        with open(path, "wb") as f:
            f.write(buf.tobytes())
        want = cv2.imread(path, cv2.IMREAD_GRAYSCALE)
        got = pkg.read_image(path)
        assert got.shape == want.shape, (name, k)
        assert np.array_equal(got, want), (name, k, int((got != want).sum()))


def test_jpeg_exif_orientation(tmp_path):
    cv2 = pytest.importorskip("cv2")
    pkg = package()
    rng = np.random.default_rng(12)
    img = rng.integers(0, 256, size=(13, 21, 3)).astype(np.uint8)
    ok, buf = cv2.imencode(".jpg", img, [cv2.IMWRITE_JPEG_QUALITY, 90])
    base = buf.tobytes()
    for little in (True, False):
        e = "<" if little else ">"
        for o in range(1, 9):
            tiff = ((b"II" if little else b"MM") + struct.pack(e + "HI", 42, 8)
                    + struct.pack(e + "H", 1)
                    + struct.pack(e + "HHIHH", 0x0112, 3, 1, o, 0)
                    + struct.pack(e + "I", 0))
            payload = b"Exif\0\0" + tiff
            app1 = b"\xff\xe1" + struct.pack(">H", len(payload) + 2) + payload
            path = str(tmp_path / f"o{o}{int(little)}.jpg")
            with open(path, "wb") as f:
                f.write(base[:2] + app1 + base[2:])
            want = cv2.imread(path, cv2.IMREAD_GRAYSCALE)
            got = pkg.read_image(path)
            assert got.shape == want.shape, (o, little)
            assert np.array_equal(got, want), (o, little)


def test_jpeg_progressive_variants(tmp_path):
    """Progressive files with restart intervals, chroma subsampling and
    qualities from 10 to 100 (spectral selection and successive
    approximation scans, end-of-band runs)."""
    cv2 = pytest.importorskip("cv2")
    pkg = package()
    rng = np.random.default_rng(14)
    k = 0
    for img in _jpeg_inputs(rng):
        for q in (10, 60, 100):
            for extra in ([], [cv2.IMWRITE_JPEG_RST_INTERVAL, 2],
                          [cv2.IMWRITE_JPEG_SAMPLING_FACTOR,
                           cv2.IMWRITE_JPEG_SAMPLING_FACTOR_420]):
                ok, buf = cv2.imencode(".jpg", img,
                                       [cv2.IMWRITE_JPEG_PROGRESSIVE, 1,
                                        cv2.IMWRITE_JPEG_QUALITY, q] + extra)
                path = str(tmp_path / f"p{k}.jpg")
                k += 1
                with open(path, "wb") as f:
                    f.write(buf.tobytes())
                want = cv2.imread(path, cv2.IMREAD_GRAYSCALE)
                got = pkg.read_image(path)
                assert got.shape == want.shape, (k, q, extra)
                assert np.array_equal(got, want), (k, q, extra,
                                                   int((got != want).sum()))


def test_jpeg_refusals(tmp_path):
    cv2 = pytest.importorskip("cv2")
    pkg = package()
    rng = np.random.default_rng(13)
    img = rng.integers(0, 256, size=(40, 40, 3)).astype(np.uint8)
    ok, base = cv2.imencode(".jpg", img)
    # (A progressive file cut between scans is a valid, less refined image.)
    files = {"truncated": base.tobytes()[:len(base) // 2],
             "no_frame": b"\xff\xd8\xff\xd9"}
    for name, data in files.items():
        p = tmp_path / f"{name}.jpg"
        p.write_bytes(data)
        with pytest.raises(pkg.SparseSeamError):
            pkg.read_image(str(p))


# ---- TIFF -------------------------------------------------------------------

def _packbits(raw: bytes) -> bytes:
    out = bytearray()
    i = 0
    while i < len(raw):
        j = i
        while j + 1 < len(raw) and raw[j + 1] == raw[i] and j - i < 127:
            j += 1
        if j > i:
            out += bytes([(257 - (j - i + 1)) & 0xFF, raw[i]])
            i = j + 1
        else:
            k = i
            while (k + 1 < len(raw) and k - i < 127 and
                   not (k + 2 < len(raw) and raw[k + 1] == raw[k + 2])):
                k += 1
            out += bytes([k - i]) + raw[i:k + 1]
            i = k + 1
    return bytes(out)


def write_tiff(path, rows, width, height, spp, bps, photometric,
               compression=1, colormap=None, predictor=1, rows_per_strip=None,
               tile=None, little=True, extra=()):
    """A one-image TIFF: `rows` are the packed sample bytes of each image row
    (top first; after differencing when predictor is 2).  `tile` = (tw, th)
    writes tiles (padded with zeros) instead of strips."""
    e = "<" if little else ">"
    row_bytes = (width * spp * bps + 7) // 8

    def pack(block: bytes) -> bytes:
        if compression == 8:
            return zlib.compress(block)
        if compression == 32773:
            return b"".join(_packbits(block[k:k + bw_bytes])
                            for k in range(0, len(block), bw_bytes))
        return block

    blocks = []
    if tile:
        tw, th = tile
        bw_bytes = (tw * spp * bps + 7) // 8
        for ty in range(0, height, th):
            for tx in range(0, width, tw):
                block = bytearray()
                for y in range(ty, ty + th):
                    r = rows[y] if y < height else bytes(row_bytes)
                    part = r[tx * spp * bps // 8:(tx + tw) * spp * bps // 8]
                    block += part + bytes(bw_bytes - len(part))
                blocks.append(pack(bytes(block)))
    else:
        bw_bytes = row_bytes
        rps = rows_per_strip or height
        for y0 in range(0, height, rps):
            blocks.append(pack(b"".join(rows[y0:y0 + rps])))
    entries = [(256, 4, [width]), (257, 4, [height]), (258, 3, [bps] * spp),
               (259, 3, [compression]), (262, 3, [photometric]),
               (277, 3, [spp]), (284, 3, [1])]
    if tile:
        entries += [(322, 3, [tile[0]]), (323, 3, [tile[1]])]
    else:
        entries.append((278, 4, [rows_per_strip or height]))
    if predictor != 1:
        entries.append((317, 3, [predictor]))
    if colormap is not None:
        entries.append((320, 3, [int(v) for v in colormap]))
    entries += list(extra)
    out = bytearray((b"II" if little else b"MM") + struct.pack(e + "HI", 42, 0))
    offsets = []
    for b in blocks:
        offsets.append(len(out))
        out += b + (b"\0" if len(b) % 2 else b"")
    entries += [(324 if tile else 273, 4, offsets),
                (325 if tile else 279, 4, [len(b) for b in blocks])]
    entries.sort()
    far = {}
    for tag, typ, vals in entries:
        fmt = "H" if typ == 3 else "I"
        if struct.calcsize(fmt) * len(vals) > 4:
            far[tag] = len(out)
            out += struct.pack(e + fmt * len(vals), *vals)
    ifd = len(out)
    out += struct.pack(e + "H", len(entries))
    for tag, typ, vals in entries:
        fmt = "H" if typ == 3 else "I"
        if tag in far:
            out += struct.pack(e + "HHII", tag, typ, len(vals), far[tag])
        else:
            v = struct.pack(e + fmt * len(vals), *vals)
            out += struct.pack(e + "HHI", tag, typ, len(vals)) + v
            out += bytes(4 - len(v))
    out += struct.pack(e + "I", 0)
    out[4:8] = struct.pack(e + "I", ifd)
    with open(path, "wb") as f:
        f.write(bytes(out))


def _tiff_cases(rng):
    """(name, writer kwargs, rows) for a spread of layouts and kinds."""
    h, w = 37, 29
    g8 = rng.integers(0, 256, size=(h, w)).astype(np.uint8)
    rows8 = [g8[y].tobytes() for y in range(h)]
    diff = np.concatenate([g8[:, :1], np.diff(g8.astype(np.int16), axis=1)],
                          axis=1).astype(np.uint8)
    rowsd = [diff[y].tobytes() for y in range(h)]
    g16 = rng.integers(0, 65536, size=(h, w)).astype(np.uint16)
    rgb = rng.integers(0, 256, size=(h, w, 3)).astype(np.uint8)
    rgba = rng.integers(0, 256, size=(h, w, 4)).astype(np.uint8)
    ga = rng.integers(0, 256, size=(h, w, 2)).astype(np.uint8)
    bits = rng.integers(0, 2, size=(h, w))
    rows1 = []
    for y in range(h):
        s = "".join(str(int(b)) for b in bits[y]) + "0" * (-w % 8)
        rows1.append(bytes(int(s[i:i + 8], 2) for i in range(0, len(s), 8)))
    cmap = rng.integers(0, 65536, size=3 * 256)
    base = dict(width=w, height=h)
    yield "gray8", dict(base, spp=1, bps=8, photometric=1), rows8
    yield "gray8_strips_packbits", dict(base, spp=1, bps=8, photometric=1,
                                        compression=32773,
                                        rows_per_strip=5), rows8
    yield "gray8_deflate_pred", dict(base, spp=1, bps=8, photometric=1,
                                     compression=8, predictor=2,
                                     rows_per_strip=7), rowsd
    yield "gray8_tiles", dict(base, spp=1, bps=8, photometric=1,
                              tile=(16, 16)), rows8
    yield "gray8_tiles_deflate", dict(base, spp=1, bps=8, photometric=1,
                                      tile=(16, 32), compression=8), rows8
    yield "gray8_big_endian", dict(base, spp=1, bps=8, photometric=1,
                                   little=False), rows8
    yield "miniswhite8", dict(base, spp=1, bps=8, photometric=0), rows8
    for little in (True, False):
        yield f"gray16_{little}", dict(base, spp=1, bps=16, photometric=1,
                                       little=little), [
            g16[y].astype("<u2" if little else ">u2").tobytes()
            for y in range(h)]
    yield "miniswhite16", dict(base, spp=1, bps=16, photometric=0), [
        g16[y].astype("<u2").tobytes() for y in range(h)]
    yield "bilevel", dict(base, spp=1, bps=1, photometric=1), rows1
    yield "bilevel_white", dict(base, spp=1, bps=1, photometric=0), rows1
    yield "gray_alpha", dict(base, spp=2, bps=8, photometric=1,
                             extra=[(338, 3, [2])]), [
        ga[y].tobytes() for y in range(h)]
    yield "rgb", dict(base, spp=3, bps=8, photometric=2), [
        rgb[y].tobytes() for y in range(h)]
    yield "rgb_tiles_packbits", dict(base, spp=3, bps=8, photometric=2,
                                     tile=(16, 16), compression=32773), [
        rgb[y].tobytes() for y in range(h)]
    for es in (0, 1, 2):
        yield f"rgba_es{es}", dict(base, spp=4, bps=8, photometric=2,
                                   extra=[(338, 3, [es])]), [
            rgba[y].tobytes() for y in range(h)]
    yield "palette", dict(base, spp=1, bps=8, photometric=3,
                          colormap=cmap), rows8
    for o in range(1, 5):
        yield f"orientation{o}", dict(base, spp=1, bps=8, photometric=1,
                                      extra=[(274, 3, [o])]), rows8
    # Orientations that swap the axes: OpenCV 4.13 reads them from square
    # images only (it fails on other shapes).
    square = [g8[y, :w].tobytes() for y in range(w)]
    for o in range(5, 9):
        yield f"orientation{o}", dict(width=w, height=w, spp=1, bps=8,
                                      photometric=1,
                                      extra=[(274, 3, [o])]), square


def test_tiff_matches_opencv(tmp_path):
    cv2 = pytest.importorskip("cv2")
    pkg = package()
    rng = np.random.default_rng(21)
    for name, kw, rows in _tiff_cases(rng):
        path = str(tmp_path / f"{name}.tif")
        write_tiff(path, rows, **kw)
        want = cv2.imread(path, cv2.IMREAD_GRAYSCALE)
        assert want is not None, name
        got = pkg.read_image(path)
        assert got.shape == want.shape, name
        assert np.array_equal(got, want), (name, int((got != want).sum()))


@pytest.mark.parametrize("compression", [1, 5, 8, 32773])
@pytest.mark.parametrize("predictor", [1, 2])
def test_tiff_written_by_opencv(tmp_path, compression, predictor):
    """LZW and the other codecs as OpenCV's own TIFF writer makes them."""
    cv2 = pytest.importorskip("cv2")
    pkg = package()
    rng = np.random.default_rng(compression + predictor)
    yy, xx = np.mgrid[0:61, 0:47]
    smooth = ((xx * 3 + yy * 5) % 256).astype(np.uint8)
    for k, img in enumerate((smooth,
                             rng.integers(0, 256, size=(61, 47, 3)).astype(
                                 np.uint8),
                             (smooth.astype(np.uint16) * 257))):
        path = str(tmp_path / f"cv{k}.tif")
        params = [cv2.IMWRITE_TIFF_COMPRESSION, compression,
                  cv2.IMWRITE_TIFF_ROWSPERSTRIP, 8]
        if predictor == 2 and compression in (5, 8):
            params += [cv2.IMWRITE_TIFF_PREDICTOR, 2]
        assert cv2.imwrite(path, img, params)
        want = cv2.imread(path, cv2.IMREAD_GRAYSCALE)
        got = pkg.read_image(path)
        assert got.shape == want.shape, k
        assert np.array_equal(got, want), (k, int((got != want).sum()))


def test_tiff_refusals(tmp_path):
    pkg = package()
    rng = np.random.default_rng(3)
    rgb16 = rng.integers(0, 65536, size=(8, 8, 3)).astype("<u2")
    cases = {
        "rgb16": (dict(width=8, height=8, spp=3, bps=16, photometric=2),
                  [rgb16[y].tobytes() for y in range(8)]),
        "gray4": (dict(width=8, height=8, spp=1, bps=4, photometric=1),
                  [bytes(4)] * 8),
        "jpeg": (dict(width=8, height=8, spp=1, bps=8, photometric=1,
                      compression=7), [bytes(8)] * 8),
    }
    for name, (kw, rows) in cases.items():
        path = str(tmp_path / f"{name}.tif")
        write_tiff(path, rows, **kw)
        with pytest.raises(pkg.SparseSeamError):
            pkg.read_image(path)
    cut = tmp_path / "cut.tif"
    write_tiff(str(cut), [bytes(range(8))] * 8, width=8, height=8, spp=1,
               bps=8, photometric=1)
    data = cut.read_bytes()
    cut.write_bytes(data[:20])
    with pytest.raises(pkg.SparseSeamError):
        pkg.read_image(str(cut))
