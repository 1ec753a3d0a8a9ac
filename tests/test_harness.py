"""The command-line harness (the reference's CLI and CSV columns over the C
ABI): argument checks on the CPU; a run over image files on the GPU."""
import csv
import shutil
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT, package

HARNESS = os.path.join(ROOT, "sparse-seam_b200", "ss_harness")
COLUMNS = ("algorithm,image,width,height,megapixels,warmup,repetitions,"
           "block,total_allocated_bytes,total_allocated_Bpp,"
           "auxiliary_bytes,auxiliary_Bpp,"
           "median_compute_ms,p95_compute_ms,compute_mpix_s,"
           "median_h2h_ms,p95_h2h_ms,h2h_mpix_s,"
           "median_iterations,p95_iterations,"
           "oracle_max_mismatches,oracle_min_mismatches,"
           "cross_max_mismatches,cross_min_mismatches").split(",")


def run(*args, timeout=600):
    return subprocess.run([HARNESS, *args], capture_output=True, text=True,
                          timeout=timeout)


def test_usage_errors_need_no_gpu(tmp_path):
    package()   # builds nothing, but fails loudly if the library is missing
    assert os.path.exists(HARNESS)
    assert run().returncode == 2
    assert run(str(tmp_path)).returncode == 2                  # no --output
    assert run(str(tmp_path), f"--output={tmp_path}",
               f"--expected-max={tmp_path}").returncode == 2   # max w/o min
    assert run(str(tmp_path), f"--output={tmp_path}",
               "--reps=0").returncode == 2
    assert run(str(tmp_path), f"--output={tmp_path}",
               "--tile=24").returncode == 2
    assert run(str(tmp_path), f"--output={tmp_path}",
               "--bogus").returncode == 2


@pytest.mark.gpu
def test_harness_over_image_files(tmp_path, golden_cases):
    pkg = package()
    images = tmp_path / "in"
    emax = tmp_path / "max"
    emin = tmp_path / "min"
    for d in (images, emax, emin):
        d.mkdir()
    picked = [c for c in golden_cases if c.image.size >= 30][:6]
    for c in picked:
        pkg.write_pgm(str(images / f"{c.name}.pgm"), c.image)
        pkg.write_pgm(str(emax / f"{c.name}.pgm"), c.maxima)
        pkg.write_pgm(str(emin / f"{c.name}.pgm"), c.minima)
    rng = np.random.default_rng(3)
    big = (rng.integers(0, 256, size=(300, 517)) >> 4 << 4).astype(np.uint8)
    pkg.write_pgm(str(images / "zz_big.pgm"), big)
    want = oracle.extrema(big)
    pkg.write_pgm(str(emax / "zz_big.pgm"), want[0])
    pkg.write_pgm(str(emin / "zz_big.pgm"), want[1])
    out = tmp_path / "out"
    r = run(str(images), f"--output={out}", f"--expected-max={emax}",
            f"--expected-min={emin}", "--warmup=1", "--reps=3", "--masks")
    assert r.returncode == 0, r.stdout + r.stderr
    with open(out / "ss_harness.csv", newline="") as f:
        rows = list(csv.DictReader(f))
    assert list(rows[0].keys()) == COLUMNS
    assert len(rows) == len(picked) + 1
    for row in rows:
        for k in ("oracle_max_mismatches", "oracle_min_mismatches",
                  "cross_max_mismatches", "cross_min_mismatches"):
            assert row[k] == "0", row
        assert float(row["median_compute_ms"]) > 0
    assert (out / "environment.txt").exists()
    got = pkg.read_image(str(out / "masks" / "zz_big_max.pgm"))
    assert np.array_equal(got, want[0])


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_percentiles_interpolate_like_the_reference(tmp_path):
    """median / p95 columns: linear interpolation at q * (n - 1)
    (harness/primary/gpu_common_v0_6.cu:86-103), pinned on even-length
    samples where nearest-rank would differ."""
    exe = str(tmp_path / "percentile_check")
    subprocess.check_call([
        "g++", "-O2", "-std=c++17",
        "-I" + os.path.join(ROOT, "sparse-seam_b200", "csrc"), "-o", exe,
        os.path.join(ROOT, "tests", "native", "percentile_check.cpp")])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.strip() == "OK", out.stdout
