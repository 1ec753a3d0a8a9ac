"""The serving loop and the batch autotuner on the GPU: every result equals
the image's result alone (ss_extrema) and the oracle's, in any mix."""
import importlib

import numpy as np
import pytest

import oracle
from conftest import package

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _serve():
    return importlib.import_module("sparse-seam_b200.serve")


def _mixed_images(count, seed, lo=16, hi=600):
    synth = importlib.import_module("sparse-seam_b200.synth")
    return [t.cpu() for t in synth.uneven_batch(count, seed=seed, lo=lo, hi=hi)]


def _alone(img_cpu, tile=32):
    pkg = package()
    d = img_cpu.cuda()
    mx, mn = pkg.extrema(d, tile=tile)
    torch.cuda.synchronize()
    return mx.cpu().numpy(), mn.cpu().numpy()


def _pinned_like(t):
    return torch.empty(t.shape, dtype=torch.uint8, pin_memory=True)


@pytest.mark.parametrize("persistent,unpack", [(True, 0), (False, 3),
                                               (True, -1)],
                         ids=["persistent-compact", "grid-compact",
                              "persistent-bytes"])
def test_mix_equals_alone_host_requests(persistent, unpack):
    serve = _serve()
    images = _mixed_images(60, seed=3)
    pinned = []
    for im in images:
        p = _pinned_like(im)
        p.copy_(im)
        pinned.append(p)
    outs = [(_pinned_like(im), _pinned_like(im)) for im in images]
    with serve.Server(tile=32, persistent=persistent, inflight=3,
                      max_batch_images=16, batch_tiles=4096,
                      pool_bytes=64 << 20, unpack_threads=unpack) as srv:
        tickets = [srv.submit(pinned[i], *outs[i], user=i)
                   for i in range(len(images))]
        done = []
        while len(done) < len(images):
            done.extend(srv.poll(timeout_us=100_000))
        stats = srv.stats()
    assert sorted(int(c.ticket) for c in done) == sorted(tickets)
    assert all(c.status == 0 for c in done), \
        sorted(set(int(c.status) for c in done))
    for c in done:
        assert c.submit_ns <= c.admit_ns <= c.launch_ns <= c.done_ns
    # Requests that arrived together shared batches.
    assert stats["max_batch_images_seen"] >= 2
    assert stats["completed"] == len(images)
    assert stats["pool_high_water"] <= stats["pool_bytes"]
    for i, im in enumerate(images):
        got = (outs[i][0].numpy(), outs[i][1].numpy())
        alone = _alone(im)
        want = oracle.extrema(im.numpy())
        for g, a, w in zip(got, alone, want):
            assert np.array_equal(g, a), f"request {i} differs from alone"
            assert np.array_equal(g, w), f"request {i} differs from oracle"


def test_admission_waits_for_pool_memory_and_batches_overlap():
    serve = _serve()
    synth = importlib.import_module("sparse-seam_b200.synth")
    # Each 1024x1024 request needs 3 MiB of pool: 8 MiB admits two at once.
    images = [synth.smooth_noise(1024, 1024, seed=s).cpu() for s in range(6)]
    images += [torch.from_numpy(synth.checkerboard(1024, 1024, 3))]
    pinned = []
    for im in images:
        p = _pinned_like(im)
        p.copy_(im)
        pinned.append(p)
    outs = [(_pinned_like(im), _pinned_like(im)) for im in images]
    with serve.Server(tile=32, inflight=2, max_batch_images=4,
                      batch_tiles=8192, pool_bytes=8 << 20) as srv:
        for i in range(len(images)):
            srv.submit(pinned[i], *outs[i], user=i)
        done = []
        while len(done) < len(images):
            done.extend(srv.poll(timeout_us=100_000))
        stats = srv.stats()
    assert all(c.status == 0 for c in done)
    assert stats["pool_high_water"] <= 8 << 20
    assert stats["pool_high_water"] >= 3 << 20
    for i, im in enumerate(images):
        want = oracle.extrema(im.numpy(), method="bands", threads=4)
        assert np.array_equal(outs[i][0].numpy(), want[0]), i
        assert np.array_equal(outs[i][1].numpy(), want[1]), i


def test_device_requests_and_rejections():
    serve = _serve()
    pkg = package()
    images = [t for t in importlib.import_module(
        "sparse-seam_b200.synth").uneven_batch(24, seed=8, lo=8, hi=300,
                                                device="cuda")]
    outs = [(torch.empty_like(i), torch.empty_like(i)) for i in images]
    with serve.Server(tile=32, inflight=2, max_batch_images=8,
                      batch_tiles=256, pool_bytes=1 << 20) as srv:
        for i, im in enumerate(images):
            srv.submit(im, *outs[i], device=True, user=i)
        # More tiles than one batch holds, or more bytes than the pool.
        big = torch.zeros((1024, 1024), dtype=torch.uint8)
        with pytest.raises(pkg.SparseSeamError) as e:
            srv.submit(big, big, big)
        assert e.value.status == 5
        done = []
        while len(done) < len(images):
            done.extend(srv.poll(timeout_us=100_000))
    assert all(c.status == 0 for c in done)
    for i, im in enumerate(images):
        want = oracle.extrema(im.cpu().numpy())
        assert np.array_equal(outs[i][0].cpu().numpy(), want[0]), i
        assert np.array_equal(outs[i][1].cpu().numpy(), want[1]), i


def test_poisson_trace_reports_latency():
    serve = _serve()
    images = _mixed_images(16, seed=11, lo=64, hi=512)
    pinned = []
    for im in images:
        p = _pinned_like(im)
        p.copy_(im)
        pinned.append(p)
    outs = [(_pinned_like(im), _pinned_like(im)) for im in images]
    arrivals = serve.poisson_trace(400.0, 0.25, seed=1)
    with serve.Server(tile=32, inflight=2, batch_tiles=4096,
                      pool_bytes=64 << 20) as srv:
        res = serve.run_trace(
            srv, arrivals,
            lambda i: (pinned[i % 16], *outs[i % 16]))
    assert res.requests == len(arrivals) and res.failures == 0
    assert 0 < res.p50_ms <= res.p99_ms <= res.max_ms
    for i, im in enumerate(images[:4]):
        want = oracle.extrema(im.numpy())
        assert np.array_equal(outs[i][0].numpy(), want[0])


def test_autotuned_batch_matches_oracle():
    at = importlib.import_module("sparse-seam_b200.autotune")
    synth = importlib.import_module("sparse-seam_b200.synth")
    choices = [c for c in at.candidates()
               if (c.tile == 32 and c.group in (0, 4)) or
               (c.tile in (16, 64) and not c.persistent)]
    assert {c.flatten for c in choices} == {0, 1, 2}
    table = at.tune(pixels_per_class=1 << 19, reps=1, classes=(0, 1, 2, 3),
                    choices=choices, mix_images=24)
    assert set(table.choices) == {0, 1, 2, 3}
    assert table.mix in choices
    images = synth.uneven_batch(40, seed=21, lo=16, hi=900, device="cuda")
    maxs = [torch.empty_like(i) for i in images]
    mins = [torch.empty_like(i) for i in images]
    tb = at.TunedBatch(images, maxs, mins, table)
    wants = [oracle.extrema(im.cpu().numpy()) for im in images]
    assert tb.form in tb.timings_ms
    mix = table.mix
    whole = pkg_plan = None
    import importlib as _il
    pkg = _il.import_module("sparse-seam_b200")
    pkg_plan = pkg.BatchPlan(images, maxs, mins, tile=mix.tile)
    whole = pkg_plan.make_workspace()
    # The form `run` picked, the split by size class itself, and one launch
    # with the mix's choice.
    for form in (tb.run,
                 lambda: tb._run_parts(torch.cuda.current_stream()),
                 lambda: pkg_plan.run_launch(whole, warps=mix.warps,
                                             persistent=mix.persistent,
                                             group=mix.group,
                                             flatten=mix.flatten)):
        for m in maxs + mins:
            m.fill_(5)
        form()
        torch.cuda.synchronize()
        for part in tb.parts:
            part[2].read_status()
        whole.read_status()
        for i, want in enumerate(wants):
            assert np.array_equal(maxs[i].cpu().numpy(), want[0]), i
            assert np.array_equal(mins[i].cpu().numpy(), want[1]), i


@pytest.mark.parametrize("group", [1, 2, 8, 32])
def test_seam_resolve_grouping_is_exact(group):
    pkg = package()
    synth = importlib.import_module("sparse-seam_b200.synth")
    images = synth.uneven_batch(30, seed=group, lo=16, hi=700, device="cuda")
    maxs = [torch.empty_like(i) for i in images]
    mins = [torch.empty_like(i) for i in images]
    plan = pkg.BatchPlan(images, maxs, mins, tile=32)
    ws = plan.make_workspace()
    for persistent in (False, True):
        for m in maxs + mins:
            m.fill_(7)
        plan.run_launch(ws, warps=-4, persistent=persistent, group=group)
        ws.read_status()
        for i, im in enumerate(images):
            want = oracle.extrema(im.cpu().numpy())
            assert np.array_equal(maxs[i].cpu().numpy(), want[0]), i
            assert np.array_equal(mins[i].cpu().numpy(), want[1]), i


def test_large_requests_come_back_compact():
    """Requests of 8 Mpixel and more take the bit-plane read-back; their
    masks equal the oracle's like the small ones."""
    serve = _serve()
    synth = importlib.import_module("sparse-seam_b200.synth")
    images = [synth.smooth_noise(2048, 4096, seed=s).cpu() for s in range(2)]
    images.append(torch.from_numpy(synth.quantize(
        synth.uniform_q16(2900, 2900, 5), 4)))
    images.append(torch.from_numpy(synth.uniform_q16(300, 200, 6)))
    pinned = []
    for im in images:
        p = _pinned_like(im)
        p.copy_(im)
        pinned.append(p)
    outs = [(_pinned_like(im), _pinned_like(im)) for im in images]
    with serve.Server(tile=32, inflight=2, batch_tiles=1 << 15,
                      pool_bytes=256 << 20) as srv:
        for i in range(len(images)):
            srv.submit(pinned[i], *outs[i], user=i)
        done = []
        while len(done) < len(images):
            done.extend(srv.poll(timeout_us=100_000))
    assert all(c.status == 0 for c in done)
    for i, im in enumerate(images):
        want = oracle.extrema(im.numpy(), method="bands", threads=8)
        assert np.array_equal(outs[i][0].numpy(), want[0]), i
        assert np.array_equal(outs[i][1].numpy(), want[1]), i


def test_served_files_match_oracle(tmp_path):
    """Image files decoded by the library straight into pinned buffers and
    served: every result equals the oracle's on the decoded pixels."""
    serve = importlib.import_module("sparse-seam_b200.serve")
    synth = importlib.import_module("sparse-seam_b200.synth")
    pkg = package()
    rng = np.random.default_rng(31)
    paths = []
    for i, (h, w) in enumerate([(321, 481), (700, 1029), (64, 64),
                                (1356, 2040)]):
        img = synth.quantize(synth.smooth_noise_np(h, w, 40 + i),
                             int(rng.integers(2, 257)))
        p = tmp_path / f"img_{i}.pgm"
        pkg.write_pgm(str(p), img)
        paths.append(str(p))
    cv2 = pytest.importorskip("cv2")
    img = synth.smooth_noise_np(500, 333, 77)
    p = tmp_path / "img_png.png"
    assert cv2.imwrite(str(p), img)
    paths.append(str(p))
    with serve.Server(tile=32, inflight=2, max_batch_images=8,
                      batch_tiles=1 << 14, pool_bytes=64 << 20) as srv:
        out = serve.serve_files(srv, paths)
    for path in paths:
        want = oracle.extrema(pkg.read_image(path))
        mx, mn = out[path]
        assert np.array_equal(mx.numpy(), want[0]), path
        assert np.array_equal(mn.numpy(), want[1]), path
