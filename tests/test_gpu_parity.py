"""Bit-exact parity of the CUDA route with the CPU oracle and the golden masks.

Every test here calls the sm_100a library through its C ABI (via the package's
ctypes binding).  Masks are bytes, so the bar is exact equality.
"""
import numpy as np
import pytest

import oracle
from conftest import package

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TILES = (16, 32, 64)
# (tile, kernel configuration): every kernel family the library ships.
CONFIGS = [(16, 4), (16, 2), (32, -2), (32, -4), (32, 8), (64, -4), (64, 16),
           (64, 8)]


@pytest.fixture
def kernel_config(request):
    """Selects a kernel configuration for the test and restores the default."""
    pkg = package()
    tile, warps = request.param
    before = pkg.get_kernel_config(tile)
    pkg.set_kernel_config(tile, warps)
    yield tile
    pkg.set_kernel_config(tile, before)


def run_gpu(image: np.ndarray, tile: int, pitch_pad: int = 0,
            out_pad: int = 0, ws=None):
    pkg = package()
    h, w = image.shape
    dev = torch.device("cuda")
    if pitch_pad:
        buf = torch.full((h, w + pitch_pad), 77, dtype=torch.uint8, device=dev)
        buf[:, :w] = torch.from_numpy(image).to(dev)
        d_img = buf[:, :w]
    else:
        d_img = torch.from_numpy(np.ascontiguousarray(image)).to(dev)
    if out_pad:
        mxb = torch.full((h, w + out_pad), 9, dtype=torch.uint8, device=dev)
        mnb = torch.full((h, w + out_pad), 9, dtype=torch.uint8, device=dev)
        mx, mn = mxb[:, :w], mnb[:, :w]
    else:
        mx = mn = None
    mx, mn = pkg.extrema(d_img, tile=tile, maxima=mx, minima=mn,
                         workspace=ws)
    torch.cuda.synchronize()
    out = (mx.cpu().numpy(), mn.cpu().numpy())
    if out_pad:
        assert (mxb[:, w:] == 9).all() and (mnb[:, w:] == 9).all(), \
            "wrote outside the output rows"
    return out


def assert_same(got, want, what):
    gmx, gmn = got
    wmx, wmn = want
    if not np.array_equal(gmx, wmx) or not np.array_equal(gmn, wmn):
        raise AssertionError(
            f"{what}: {int((gmx != wmx).sum())} maxima and "
            f"{int((gmn != wmn).sum())} minima pixels differ")


@pytest.mark.parametrize("kernel_config", CONFIGS, indirect=True,
                         ids=[f"T{t}w{w}" for t, w in CONFIGS])
def test_golden_cases(golden_cases, kernel_config):
    pkg = package()
    tile = kernel_config
    for c in golden_cases:
        h, w = c.image.shape
        ws = pkg.Workspace.for_image(w, h, tile)
        got = run_gpu(c.image, tile, ws=ws)
        stats = ws.read_status()
        assert_same(got, (c.maxima, c.minima), f"{c} T={tile}")
        assert int((got[0] != 0).sum()) == c.manifest_max
        assert int((got[1] != 0).sum()) == c.manifest_min
        frag = int(oracle.tile_fragments(c.image, tile).sum())
        if pkg.get_kernel_config(tile) > 0:
            # CTA-per-tile kernels: one fragment per seam-touching tile-local
            # zone, the reference's tile_fragment_counts.
            assert stats.active_fragments == frag, (c, tile)
        else:
            # Row-scan kernels: only seam zones whose verdict can change.
            assert stats.active_fragments <= frag, (c, tile)


@pytest.mark.parametrize("kernel_config", CONFIGS, indirect=True,
                         ids=[f"T{t}w{w}" for t, w in CONFIGS])
def test_random_images_against_oracle(kernel_config):
    tile = kernel_config
    rng = np.random.default_rng(1000 + tile)
    for trial in range(40):
        h = int(rng.integers(1, 300))
        w = int(rng.integers(1, 300))
        levels = int(rng.choice([2, 3, 4, 8, 16, 64, 256]))
        img = rng.integers(0, levels, size=(h, w)).astype(np.uint8)
        got = run_gpu(img, tile, pitch_pad=int(rng.integers(0, 3)) * 13,
                      out_pad=int(rng.integers(0, 2)) * 5)
        assert_same(got, oracle.extrema(img), f"trial {trial} {h}x{w} q{levels}")


def test_config1_uniform_q16_and_constant():
    synth = pytest.importorskip("importlib").import_module(
        "sparse-seam_b200.synth")
    for img in (synth.uniform_q16(512, 512, 0), synth.constant(512, 512, 128)):
        want = oracle.extrema(img)
        for tile in TILES:
            assert_same(run_gpu(img, tile), want, f"config1 T={tile}")
    c = synth.constant(512, 512, 128)
    got = run_gpu(c, 32)
    assert (got[0] == 255).all() and (got[1] == 255).all()


@pytest.mark.parametrize("kernel_config", [(32, -2), (32, -4), (32, 8), (64, -4)],
                         indirect=True,
                         ids=["rowscan2", "rowscan4", "cta", "rowscan64"])
def test_plateau_and_seam_heavy_families(kernel_config):
    import importlib
    synth = importlib.import_module("sparse-seam_b200.synth")
    imgs = {
        "ellipse_edt": synth.ellipse_edt(1024, 1024, 3),
        "serpentine": synth.serpentine(1024, 1024),
        "spiral": synth.spiral(1024, 1024),
        "blocks": synth.blocks(1024, 1024, 8, 0, 5),
        "blocks_shift16": synth.blocks(1024, 1024, 8, 16, 5),
        "checker1": synth.checkerboard(1024, 1024, 1),
        "checker3": synth.checkerboard(1024, 1024, 3),
        "checker17": synth.checkerboard(1024, 1024, 17),
    }
    for name, img in imgs.items():
        want = oracle.extrema(img)
        for tile in TILES:
            assert_same(run_gpu(img, tile), want, f"{name} T={tile}")


def test_smooth_noise_quantization_sweep_full_size():
    import importlib
    synth = importlib.import_module("sparse-seam_b200.synth")
    base = synth.smooth_noise(1356, 2040, seed=11, device="cuda").cpu().numpy()
    for levels in (256, 64, 16, 4, 2):
        img = synth.quantize(base, levels)
        want = oracle.extrema(img, method="bands", threads=8)
        for tile in TILES:
            assert_same(run_gpu(img, tile), want, f"smooth q{levels} T={tile}")


def test_repeatable_and_workspace_reuse_across_geometries():
    pkg = package()
    rng = np.random.default_rng(5)
    ws = pkg.Workspace(max(pkg.workspace_bytes(700, 700, t) for t in TILES))
    imgs = [rng.integers(0, 4, size=s).astype(np.uint8)
            for s in [(700, 700), (33, 650), (512, 97), (700, 700)]]
    for rep in range(3):
        for img in imgs:
            for tile in TILES:
                got = run_gpu(img, tile, ws=ws)
                ws.read_status()
                assert_same(got, oracle.extrema(img), f"rep {rep} T={tile}")


@pytest.mark.parametrize("persistent", [False, True])
@pytest.mark.parametrize("tile", TILES)
def test_batch_equals_single(persistent, tile):
    import importlib
    pkg = package()
    synth = importlib.import_module("sparse-seam_b200.synth")
    images = synth.uneven_batch(48, seed=tile, lo=16, hi=400, device="cuda")
    maxs, mins = pkg.extrema_batch(images, tile=tile, persistent=persistent)
    for i, im in enumerate(images):
        host = im.cpu().numpy()
        want = oracle.extrema(host)
        assert_same((maxs[i].cpu().numpy(), mins[i].cpu().numpy()), want,
                    f"batch image {i} {host.shape}")


def test_batch_replay_is_stable():
    import importlib
    pkg = package()
    synth = importlib.import_module("sparse-seam_b200.synth")
    images = synth.uneven_batch(32, seed=9, lo=64, hi=512, device="cuda")
    maxs = [torch.empty_like(i) for i in images]
    mins = [torch.empty_like(i) for i in images]
    plan = pkg.BatchPlan(images, maxs, mins, tile=32)
    ws = plan.make_workspace()
    plan.run(ws, persistent=True)
    ws.read_status()
    first = [(a.clone(), b.clone()) for a, b in zip(maxs, mins)]
    for rep in range(5):
        for m in maxs + mins:
            m.fill_(3)
        plan.run(ws, persistent=bool(rep % 2))
        ws.read_status()
        for (a, b), mx, mn in zip(first, maxs, mins):
            assert torch.equal(a, mx) and torch.equal(b, mn)


def test_uninitialized_workspace_is_reported():
    pkg = package()
    img = torch.zeros((64, 64), dtype=torch.uint8, device="cuda")
    ws = pkg.Workspace(pkg.workspace_bytes(64, 64, 32))
    ws.buffer.zero_()  # wipes the header written by init
    with pytest.raises(pkg.SparseSeamError) as e:
        pkg.extrema(img, tile=32, workspace=ws, check=True)
    assert e.value.status == 11


@pytest.mark.parametrize("kernel_config", [(32, -2), (32, 8), (16, 4),
                                           (64, 16), (64, -4)], indirect=True,
                         ids=["rowscan", "cta32", "cta16", "cta64",
                              "rowscan64"])
def test_quantisation_fused_into_the_load(kernel_config):
    """ss_extrema_levels on the original image gives the masks of the
    re-quantised image (the reference's rule, applied on the host there)."""
    import importlib
    pkg = package()
    synth = importlib.import_module("sparse-seam_b200.synth")
    tile = kernel_config
    base = synth.smooth_noise(333, 517, seed=17, device="cuda")
    host = base.cpu().numpy()
    for levels in (2, 3, 4, 16, 64, 255, 256):
        want = oracle.extrema(synth.quantize(host, levels))
        mx, mn = pkg.extrema(base, tile=tile, levels=levels, check=True)
        assert_same((mx.cpu().numpy(), mn.cpu().numpy()), want,
                    f"levels {levels} T={tile}")


def test_quantisation_per_image_in_a_batch():
    import importlib
    pkg = package()
    synth = importlib.import_module("sparse-seam_b200.synth")
    images = synth.uneven_batch(12, seed=4, lo=20, hi=300, device="cuda")
    levels = [2, 4, 8, 16, 32, 64, 128, 256, 0, 3, 5, 7]
    maxs = [torch.empty_like(i) for i in images]
    mins = [torch.empty_like(i) for i in images]
    for persistent in (False, True):
        plan = pkg.BatchPlan(images, maxs, mins, tile=32, levels=levels)
        ws = plan.make_workspace()
        plan.run(ws, persistent=persistent)
        ws.read_status()
        for i, im in enumerate(images):
            want = oracle.extrema(synth.quantize(im.cpu().numpy(),
                                                 levels[i] or 256))
            assert_same((maxs[i].cpu().numpy(), mins[i].cpu().numpy()), want,
                        f"image {i} levels {levels[i]}")


@pytest.mark.parametrize("kernel_config", [(32, -2), (32, -4), (64, -4)],
                         indirect=True,
                         ids=["rowscan2", "rowscan4", "rowscan64"])
def test_every_store_width(kernel_config):
    """Whole-row mask stores and read-merge-writes at 16, 8, 4 and 1 bytes:
    the output pitch (and base) picks the width, the content has dense live
    tiles (long runs across seams) and sparse ones."""
    import importlib
    synth = importlib.import_module("sparse-seam_b200.synth")
    pkg = package()
    tile = kernel_config
    dev = torch.device("cuda")
    rng = np.random.default_rng(77)
    contents = {
        "blocks": synth.blocks(257, 600, 8, 16, 3),
        "q2": synth.quantize(synth.smooth_noise_np(257, 600, 5), 2),
        "natural": synth.smooth_noise_np(257, 600, 6),
        "serpentine": synth.serpentine(257, 600),
    }
    for name, img in contents.items():
        want = oracle.extrema(img)
        h, w = img.shape
        d_img = torch.from_numpy(np.ascontiguousarray(img)).to(dev)
        for pitch, shift in ((640, 0), (616, 0), (604, 0), (601, 0),
                             (640, 8), (640, 4), (640, 1)):
            base_mx = torch.full((h * pitch + 64,), 9, dtype=torch.uint8,
                                 device=dev)
            base_mn = torch.full((h * pitch + 64,), 9, dtype=torch.uint8,
                                 device=dev)
            mx = base_mx[shift:shift + h * pitch].view(h, pitch)[:, :w]
            mn = base_mn[shift:shift + h * pitch].view(h, pitch)[:, :w]
            pkg.extrema(d_img, tile=tile, maxima=mx, minima=mn, check=True)
            assert_same((mx.cpu().numpy(), mn.cpu().numpy()), want,
                        f"{name} pitch {pitch} shift {shift}")
            # Bytes between the rows are left alone.
            pad = base_mx[shift:shift + h * pitch].view(h, pitch)[:, w:]
            assert (pad == 9).all(), f"{name} pitch {pitch}: wrote padding"


@pytest.mark.parametrize("tile", [32, 64])
def test_seam_statistics(tile):
    """The status's statistics: a constant image is one zone that crosses
    every seam (every pixel waits for the merge), a one-tile image has no
    seam, and a batch's counts are its images' sums."""
    pkg = package()
    flat = torch.full((300, 200), 77, dtype=torch.uint8, device="cuda")
    small = torch.randint(0, 256, (tile, tile), dtype=torch.uint8,
                          device="cuda")
    noisy = torch.randint(0, 4, (256, 320), dtype=torch.uint8, device="cuda")
    per = []
    for im in (flat, small, noisy):
        mx, mn = torch.empty_like(im), torch.empty_like(im)
        plan = pkg.BatchPlan([im], [mx], [mn], tile=tile)
        ws = plan.make_workspace()
        plan.run(ws)
        st = ws.read_status()
        per.append(st)
        assert st.tiles == ((im.shape[0] + tile - 1) // tile) * \
            ((im.shape[1] + tile - 1) // tile)
    assert per[0].live_pixels == flat.numel()
    assert per[0].active_fragments == per[0].tiles
    assert per[1].live_pixels == 0 and per[1].active_fragments == 0
    assert 0 < per[2].live_pixels <= noisy.numel()
    images = [flat, small, noisy]
    maxs = [torch.empty_like(i) for i in images]
    mins = [torch.empty_like(i) for i in images]
    plan = pkg.BatchPlan(images, maxs, mins, tile=tile)
    ws = plan.make_workspace()
    plan.run(ws)
    st = ws.read_status()
    assert st.live_pixels == sum(p.live_pixels for p in per)
    assert st.active_fragments == sum(p.active_fragments for p in per)
    assert st.tiles == sum(p.tiles for p in per)


@pytest.mark.parametrize("tile", [16, 32, 64])
@pytest.mark.parametrize("persistent", [False, True])
def test_one_image_plans_match_the_oracle(tile, persistent):
    """A one-image plan carries its image in the launch parameters (no
    per-tile lookup); its masks equal the oracle's, with and without the
    persistent queue, at every tile edge, and with re-quantisation."""
    import importlib
    pkg = package()
    synth = importlib.import_module("sparse-seam_b200.synth")
    for seed, (h, w) in enumerate([(1, 1), (37, 300), (301, 203)]):
        im = (synth.smooth_noise(h, w, seed, device="cuda") if h * w > 1 else
              torch.full((h, w), 9, dtype=torch.uint8, device="cuda"))
        for levels in (256, 5):
            mx, mn = torch.empty_like(im), torch.empty_like(im)
            plan = pkg.BatchPlan([im], [mx], [mn], tile=tile, levels=levels)
            ws = plan.make_workspace()
            for _ in range(2):   # the persistent queue rewinds between runs
                plan.run(ws, persistent=persistent)
            ws.read_status()
            host = im.cpu().numpy()
            if levels < 256:
                b = (host.astype(np.int32) * levels) >> 8
                host = ((b * 255 + (levels - 1) // 2) //
                        (levels - 1)).astype(np.uint8)
            assert_same((mx.cpu().numpy(), mn.cpu().numpy()),
                        oracle.extrema(host),
                        f"one-image plan {h}x{w} T={tile} L={levels}")
