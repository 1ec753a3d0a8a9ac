"""Command-line options of the benchmark (CPU only: parsing and the shapes it
derives from the library's defaults)."""
import sys

import pytest

from conftest import ROOT, package


def _bench():
    sys.path.insert(0, ROOT)
    import bench
    return bench


def test_schedule_option(monkeypatch):
    bench = _bench()
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    assert bench.parse_args().schedule == "auto"
    for choice in ("grid", "persistent"):
        monkeypatch.setattr(sys, "argv", ["bench.py", "--schedule", choice])
        assert bench.parse_args().schedule == choice
    monkeypatch.setattr(sys, "argv", ["bench.py", "--schedule", "fastest"])
    with pytest.raises(SystemExit):
        bench.parse_args()


def test_later_group_matches_the_library_rule():
    """The bench's copy of the later passes' tiles per CTA: powers of two up
    to 32, the smallest that keeps the grid within 8 CTAs per SM."""
    bench = _bench()
    assert bench._later_group(2752, 148) == 4
    assert bench._later_group(1000, 148) == 1
    assert bench._later_group(10 ** 7, 148) == 32
    for tiles in (1, 1184, 1185, 2368, 2369, 37_888, 37_889):
        g = bench._later_group(tiles, 148)
        assert g in (1, 2, 4, 8, 16, 32)
        assert g == 32 or tiles <= g * 148 * 8
        assert g == 1 or tiles > (g // 2) * 148 * 8


def test_default_tile_32_config_is_a_row_scan_family():
    pkg = package()
    cfg = pkg.get_kernel_config(32)
    assert cfg in pkg.KERNEL_CONFIGS[32]
    assert cfg == pkg.KERNEL_CONFIGS[32][0]
    assert cfg < 0
