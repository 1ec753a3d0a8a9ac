"""Mutated image files (bytes changed, cut or inserted) must come back as an
image or as SparseSeamError, never crash the process.  The decoding runs in
a child process so a crash fails the test instead of ending the run."""
import subprocess
import sys
import textwrap

import pytest

CHILD = textwrap.dedent(r'''
    import random, sys, os
    import numpy as np
    sys.path.insert(0, os.path.join(sys.argv[1], "tests"))
    sys.path.insert(0, sys.argv[1])
    from conftest import package
    import test_image_io as T
    pkg = package()
    tmp = sys.argv[2]
    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, size=(23, 31, 3)).astype(np.uint8)
    bases = {}
    T.write_bmp(tmp + "/b.bmp", [img[y].tobytes() for y in range(23)], 31, 23, 24)
    T.write_bmp(tmp + "/r.bmp", None, 31, 23, 8, comp=1,
                palette=rng.integers(0, 256, size=(256, 3)),
                stream=T.rle_stream(rng, 31, 23, False))
    T.write_tiff(tmp + "/t.tif", [img[y].tobytes() for y in range(23)],
                 width=31, height=23, spp=3, bps=8, photometric=2,
                 tile=(16, 16), compression=32773)
    T.write_tiff(tmp + "/d.tif", [img[y, :, 0].tobytes() for y in range(23)],
                 width=31, height=23, spp=1, bps=8, photometric=1,
                 compression=8, rows_per_strip=5)
    T.write_png(tmp + "/p.png", img.reshape(23, -1), 2, 8)
    for f in ("b.bmp", "r.bmp", "t.tif", "d.tif", "p.png"):
        bases[f] = open(tmp + "/" + f, "rb").read()
    bases["pgm"] = b"P5\n31 23\n255\n" + img[..., 0].tobytes()
    try:
        import cv2
        bases["jpg"] = cv2.imencode(".jpg", img,
                                    [cv2.IMWRITE_JPEG_RST_INTERVAL, 2])[1].tobytes()
    except ImportError:
        pass
    r = random.Random(int(sys.argv[3]))
    for name, base in bases.items():
        for i in range(int(sys.argv[4])):
            b = bytearray(base)
            for _ in range(r.randint(1, 8)):
                q = r.random()
                if q < 0.6 and len(b):
                    b[r.randrange(len(b))] = r.randrange(256)
                elif q < 0.8:
                    b = b[:r.randrange(len(b) + 1)]
                else:
                    p = r.randrange(len(b) + 1)
                    b[p:p] = bytes(r.randrange(256) for _ in range(r.randint(1, 16)))
            path = tmp + "/m"
            open(path, "wb").write(bytes(b))
            try:
                pkg.read_image(path)
            except pkg.SparseSeamError:
                pass
    print("fuzz ok")
''')


@pytest.mark.parametrize("seed", [1, 2])
def test_mutated_files_never_crash(tmp_path, seed):
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    proc = subprocess.run(
        [sys.executable, "-c", CHILD, root, str(tmp_path), str(seed), "300"],
        capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stderr[-2000:]
    assert "fuzz ok" in proc.stdout
