"""Host-to-host batches: pinned staging, copy/compute overlap, async read-back.

The reference times a host-to-host form per image (H2D of the image, the
route, D2H of both masks; harness/primary/gpu_common_v0_6.cu:351-373).  Here a
corpus of host images is cut into chunks; each chunk's images are packed into
one pinned buffer and copied with a single cudaMemcpyAsync on a copy stream,
run as one batch on the compute stream, and both masks come back with one
copy each on a read-back stream, so the H2D of chunk c+1, the kernels of
chunk c and the D2H of chunk c-1 overlap.
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np


class HostBatch:
    """A fixed corpus of host images processed host-to-host.

    `images` is a list of 2-D uint8 numpy arrays.  After construction the
    inputs live in pinned host memory (`self.inputs`, views per image) and
    the results land in pinned host memory (`self.maxima`, `self.minima`,
    views per image).  `run()` performs one full host -> device -> host pass.
    """

    def __init__(self, images: Sequence[np.ndarray], tile: int = 32,
                 chunks: int = 4, persistent: bool = False, device=None):
        import torch
        from importlib import import_module
        self._pkg = import_module("sparse-seam_b200")
        self.device = torch.device(device or "cuda")
        self.tile = tile
        self.persistent = persistent
        shapes = [tuple(im.shape) for im in images]
        sizes = [h * w for h, w in shapes]
        self.pixels = int(sum(sizes))
        n = len(images)
        chunks = max(1, min(chunks, n))
        # Cut into chunks of about equal pixel count.
        bounds = [0]
        target = self.pixels / chunks
        acc = 0
        for i, s in enumerate(sizes):
            acc += s
            if acc >= target * len(bounds) and len(bounds) < chunks:
                bounds.append(i + 1)
        if bounds[-1] != n:
            bounds.append(n)
        self.chunks = []
        offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        pin = dict(dtype=torch.uint8, pin_memory=True)
        self.h_in = torch.empty(self.pixels, **pin)
        self.h_max = torch.empty(self.pixels, **pin)
        self.h_min = torch.empty(self.pixels, **pin)
        h_in_np = self.h_in.numpy()
        for i, im in enumerate(images):
            h_in_np[offsets[i]:offsets[i + 1]] = np.ascontiguousarray(
                im).reshape(-1)
        self.inputs = [h_in_np[offsets[i]:offsets[i + 1]].reshape(shapes[i])
                       for i in range(n)]
        self.maxima = [self.h_max.numpy()[offsets[i]:offsets[i + 1]]
                       .reshape(shapes[i]) for i in range(n)]
        self.minima = [self.h_min.numpy()[offsets[i]:offsets[i + 1]]
                       .reshape(shapes[i]) for i in range(n)]
        self.d_in = torch.empty(self.pixels, dtype=torch.uint8,
                                device=self.device)
        self.d_max = torch.empty_like(self.d_in)
        self.d_min = torch.empty_like(self.d_in)
        ws_bytes = 0
        for c in range(len(bounds) - 1):
            a, b = bounds[c], bounds[c + 1]
            lo, hi = int(offsets[a]), int(offsets[b])
            ims = [self.d_in[offsets[i]:offsets[i + 1]].view(shapes[i])
                   for i in range(a, b)]
            mxs = [self.d_max[offsets[i]:offsets[i + 1]].view(shapes[i])
                   for i in range(a, b)]
            mns = [self.d_min[offsets[i]:offsets[i + 1]].view(shapes[i])
                   for i in range(a, b)]
            plan = self._pkg.BatchPlan(ims, mxs, mns, tile=tile)
            ws_bytes = max(ws_bytes, plan.workspace_bytes)
            self.chunks.append((lo, hi, plan))
        self.workspace = self._pkg.Workspace(ws_bytes, device=self.device)
        self.copy_in = torch.cuda.Stream(device=self.device)
        self.compute = torch.cuda.Stream(device=self.device)
        self.copy_out = torch.cuda.Stream(device=self.device)
        torch.cuda.synchronize(self.device)

    @property
    def h2d_bytes(self) -> int:
        return self.pixels

    @property
    def d2h_bytes(self) -> int:
        return 2 * self.pixels

    def run(self, start_stream=None):
        """Enqueues one host-to-host pass; returns the event that ends it.

        The pass starts after the work already queued on `start_stream`
        (torch's current stream by default) and the returned event is
        recorded on the read-back stream after the last mask copy.
        """
        import torch
        start_stream = start_stream or torch.cuda.current_stream(self.device)
        begin = torch.cuda.Event()
        begin.record(start_stream)
        self.copy_in.wait_event(begin)
        self.compute.wait_event(begin)
        self.copy_out.wait_event(begin)
        for lo, hi, plan in self.chunks:
            with torch.cuda.stream(self.copy_in):
                self.d_in[lo:hi].copy_(self.h_in[lo:hi], non_blocking=True)
                loaded = torch.cuda.Event()
                loaded.record(self.copy_in)
            self.compute.wait_event(loaded)
            plan.run(self.workspace, persistent=self.persistent,
                     stream=self.compute)
            done = torch.cuda.Event()
            done.record(self.compute)
            self.copy_out.wait_event(done)
            with torch.cuda.stream(self.copy_out):
                self.h_max[lo:hi].copy_(self.d_max[lo:hi], non_blocking=True)
                self.h_min[lo:hi].copy_(self.d_min[lo:hi], non_blocking=True)
        end = torch.cuda.Event(enable_timing=True)
        end.record(self.copy_out)
        # The next pass may reuse the device buffers only after this one.
        start_stream.wait_event(end)
        return end

    def check(self) -> None:
        """Synchronises and raises on a device-side failure."""
        import torch
        torch.cuda.synchronize(self.device)
        self.workspace.read_status(self.compute)


def run_corpus(images: Sequence[np.ndarray], tile: int = 32,
               chunks: int = 4) -> tuple:
    """One-shot host-to-host pass over host images; returns mask copies."""
    hb = HostBatch(images, tile=tile, chunks=chunks)
    hb.run()
    hb.check()
    return ([m.copy() for m in hb.maxima], [m.copy() for m in hb.minima])
