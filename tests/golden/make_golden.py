"""Packs the reference's golden regional-extrema cases into one fixture file.

The reference ships 206 golden cases as binary PGM files (an input image plus
MATLAB's 8-connected imregionalmax / imregionalmin masks), with a manifest of
per-case pixel counts:

    oracles/oracle_v0_1/                         34 designed cases
    oracles/oracle_v0_2_fuzz/                   160 fuzz cases
    oracles/oracle_v0_3_sparse_seam_adversarial/ 12 seam-adversarial cases

(builders: oracles/build_oracle_v0_1.m:31-94, build_fuzz_oracle_v0_2.m:18-76,
build_sparse_seam_adversarial_oracle_v0_3.m:17-78).  This script reads them
where they lie and writes ``oracle_cases.npz`` beside itself: images as raw
bytes, masks bit-packed, manifest counts, and the SHA-256 of every source file.
The GPU box does not have the reference tree, so the tests read only the npz.

Run:  python tests/golden/make_golden.py [--reference DIR]
"""
from __future__ import annotations

import argparse
import csv
import hashlib
import os
import sys

import numpy as np

SUITES = (
    "oracle_v0_1",
    "oracle_v0_2_fuzz",
    "oracle_v0_3_sparse_seam_adversarial",
)


def read_pgm(path: str) -> np.ndarray:
    """Reads a binary (P5) 8-bit PGM; the header is 'P5 W H 255' + one space."""
    with open(path, "rb") as handle:
        data = handle.read()
    fields = []
    pos = 0
    while len(fields) < 4:
        while data[pos:pos + 1].isspace():
            pos += 1
        if data[pos:pos + 1] == b"#":
            while data[pos:pos + 1] not in (b"\n", b""):
                pos += 1
            continue
        start = pos
        while not data[pos:pos + 1].isspace():
            pos += 1
        fields.append(data[start:pos])
    pos += 1  # the single whitespace byte after maxval
    if fields[0] != b"P5" or int(fields[3]) != 255:
        raise ValueError(f"{path}: not an 8-bit binary PGM")
    width, height = int(fields[1]), int(fields[2])
    pixels = np.frombuffer(data, dtype=np.uint8, count=width * height,
                           offset=pos)
    return pixels.reshape(height, width).copy()


def sha256(path: str) -> str:
    with open(path, "rb") as handle:
        return hashlib.sha256(handle.read()).hexdigest()


def main() -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference",
                        default=os.environ.get("SS_REFERENCE_TREE"),
                        help="reference tree (default: $SS_REFERENCE_TREE)")
    parser.add_argument(
        "--out",
        default=os.path.join(os.path.dirname(os.path.abspath(__file__)),
                             "oracle_cases.npz"))
    args = parser.parse_args()
    if not args.reference:
        parser.error("no reference tree: pass --reference DIR or set "
                     "SS_REFERENCE_TREE")

    names, suites, heights, widths = [], [], [], []
    manifest_max, manifest_min = [], []
    images, maxima, minima = [], [], []
    hashes = []
    for suite in SUITES:
        root = os.path.join(args.reference, "oracles", suite)
        with open(os.path.join(root, "oracle_manifest.csv"), newline="") as f:
            rows = list(csv.DictReader(f))
        for row in rows:
            case = row["case_id"]
            image = read_pgm(os.path.join(root, "inputs", case + ".pgm"))
            emax = read_pgm(os.path.join(root, "expected_max", case + ".pgm"))
            emin = read_pgm(os.path.join(root, "expected_min", case + ".pgm"))
            h, w = int(row["height"]), int(row["width"])
            if image.shape != (h, w) or emax.shape != (h, w) or \
                    emin.shape != (h, w):
                raise ValueError(f"{suite}/{case}: shape mismatch")
            if not set(np.unique(emax)) <= {0, 255} or \
                    not set(np.unique(emin)) <= {0, 255}:
                raise ValueError(f"{suite}/{case}: masks are not 0/255")
            names.append(case)
            suites.append(suite)
            heights.append(h)
            widths.append(w)
            manifest_max.append(int(row["max_pixels"]))
            manifest_min.append(int(row["min_pixels"]))
            images.append(image.reshape(-1))
            maxima.append(np.packbits(emax.reshape(-1) != 0))
            minima.append(np.packbits(emin.reshape(-1) != 0))
            for sub in ("inputs", "expected_max", "expected_min"):
                hashes.append(sha256(os.path.join(root, sub, case + ".pgm")))

    def offsets(chunks):
        out = np.zeros(len(chunks) + 1, dtype=np.int64)
        out[1:] = np.cumsum([len(c) for c in chunks])
        return out

    np.savez_compressed(
        args.out,
        names=np.array(names),
        suites=np.array(suites),
        heights=np.array(heights, dtype=np.int32),
        widths=np.array(widths, dtype=np.int32),
        manifest_max=np.array(manifest_max, dtype=np.int64),
        manifest_min=np.array(manifest_min, dtype=np.int64),
        image_data=np.concatenate(images),
        image_offsets=offsets(images),
        max_bits=np.concatenate(maxima),
        max_offsets=offsets(maxima),
        min_bits=np.concatenate(minima),
        min_offsets=offsets(minima),
        source_sha256=np.array(hashes).reshape(-1, 3),
    )
    print(f"wrote {len(names)} cases to {args.out} "
          f"({os.path.getsize(args.out)} bytes)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
