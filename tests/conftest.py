import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "oracle_cases.npz")


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200, sm_100a)")


def package():
    """The product package (its directory name is not a Python identifier)."""
    return importlib.import_module("sparse-seam_b200")


class GoldenCase:
    __slots__ = ("name", "suite", "image", "maxima", "minima",
                 "manifest_max", "manifest_min")

    def __repr__(self):
        return f"{self.suite}/{self.name}"


def load_golden():
    data = np.load(GOLDEN)
    cases = []
    for i, name in enumerate(data["names"]):
        h = int(data["heights"][i])
        w = int(data["widths"][i])
        n = h * w
        c = GoldenCase()
        c.name = str(name)
        c.suite = str(data["suites"][i])
        io = data["image_offsets"]
        c.image = data["image_data"][io[i]:io[i + 1]].reshape(h, w).copy()
        mo = data["max_offsets"]
        c.maxima = (np.unpackbits(data["max_bits"][mo[i]:mo[i + 1]])[:n]
                    .reshape(h, w) * 255).astype(np.uint8)
        no = data["min_offsets"]
        c.minima = (np.unpackbits(data["min_bits"][no[i]:no[i + 1]])[:n]
                    .reshape(h, w) * 255).astype(np.uint8)
        c.manifest_max = int(data["manifest_max"][i])
        c.manifest_min = int(data["manifest_min"][i])
        cases.append(c)
    return cases


@pytest.fixture(scope="session")
def golden_cases():
    return load_golden()
