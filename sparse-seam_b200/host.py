"""Host-to-host batches: pinned staging, copy/compute overlap, async read-back.

The reference times a host-to-host form per image (H2D of the image, the
route, D2H of both masks; harness/primary/gpu_common_v0_6.cu:351-373).  Here a
corpus of host images is cut into chunks; each chunk's images are packed into
one pinned buffer and copied with a single cudaMemcpyAsync on a copy stream,
and run as one batch on the compute stream.  The masks come back on a
read-back stream, so the H2D of chunk c+1, the kernels of chunk c and the D2H
of chunk c-1 overlap.  With `packed` (the default) the device packs both
masks into bit planes (ss_pack_masks), only the planes cross the bus (0.25
instead of 2 bytes per pixel), and a host function enqueued on a fourth
stream expands them into the pinned byte masks with all host threads
(ss_enqueue_unpack_masks), overlapping the transfers of the next chunks.
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
                 chunks: int = 4, persistent: bool = False, device=None,
                 packed: bool = True, threads: int = 0):
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
        self.packed = packed
        self.threads = int(threads)
        if packed:
            # Bit planes: per chunk (hi - lo + 31) // 32 words per mask.
            self.words = []
            w0 = 0
            for lo, hi, _ in self.chunks:
                n_words = (hi - lo + 31) // 32
                self.words.append((w0, n_words))
                w0 += n_words
            self.d_bits = torch.empty((2, max(w0, 1)), dtype=torch.int32,
                                      device=self.device)
            self.h_bits = torch.empty((2, max(w0, 1)), dtype=torch.int32,
                                      pin_memory=True)
            self.unpack = torch.cuda.Stream(device=self.device)
        torch.cuda.synchronize(self.device)

    @property
    def h2d_bytes(self) -> int:
        return self.pixels

    @property
    def d2h_bytes(self) -> int:
        if self.packed:
            return 2 * 4 * sum(n for _, n in self.words)
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
        if self.packed:
            self.unpack.wait_event(begin)
        lib = self._pkg.lib()
        for c, (lo, hi, plan) in enumerate(self.chunks):
            with torch.cuda.stream(self.copy_in):
                self.d_in[lo:hi].copy_(self.h_in[lo:hi], non_blocking=True)
                loaded = torch.cuda.Event()
                loaded.record(self.copy_in)
            self.compute.wait_event(loaded)
            plan.run(self.workspace, persistent=self.persistent,
                     stream=self.compute)
            if self.packed:
                w0, nw = self.words[c]
                d_mx = self.d_bits[0, w0:w0 + nw]
                d_mn = self.d_bits[1, w0:w0 + nw]
                self._pkg._check(lib.ss_pack_masks(
                    self.d_max[lo:hi].data_ptr(),
                    self.d_min[lo:hi].data_ptr(), hi - lo, d_mx.data_ptr(),
                    d_mn.data_ptr(),
                    self._pkg._stream_handle(self.compute)), "ss_pack_masks")
            done = torch.cuda.Event()
            done.record(self.compute)
            self.copy_out.wait_event(done)
            with torch.cuda.stream(self.copy_out):
                if self.packed:
                    self.h_bits[0, w0:w0 + nw].copy_(d_mx, non_blocking=True)
                    self.h_bits[1, w0:w0 + nw].copy_(d_mn, non_blocking=True)
                    arrived = torch.cuda.Event()
                    arrived.record(self.copy_out)
                else:
                    self.h_max[lo:hi].copy_(self.d_max[lo:hi],
                                            non_blocking=True)
                    self.h_min[lo:hi].copy_(self.d_min[lo:hi],
                                            non_blocking=True)
            if self.packed:
                self.unpack.wait_event(arrived)
                self._pkg._check(lib.ss_enqueue_unpack_masks(
                    self.h_bits[0, w0:].data_ptr(),
                    self.h_bits[1, w0:].data_ptr(), hi - lo,
                    self.h_max[lo:hi].data_ptr(), self.h_min[lo:hi].data_ptr(),
                    self.threads, self._pkg._stream_handle(self.unpack)),
                    "ss_enqueue_unpack_masks")
        end = torch.cuda.Event(enable_timing=True)
        end.record(self.unpack if self.packed else self.copy_out)
        # The next pass may reuse the device buffers only after this one.
        start_stream.wait_event(end)
        return end

    def tune_threads(self, stream=None, candidates=None, reps: int = 3) -> int:
        """Picks the host thread count of the mask expansion by timing.

        The expansion shares the host's memory with the copy engines' reads
        of the inputs, and how many threads pay off depends on the host and
        on what else runs there.  Times `reps` passes per candidate (by
        default a quarter, half and all but one of the processors), keeps the
        fastest in `self.threads` and returns it.
        """
        import os
        import torch
        if not self.packed:
            return self.threads
        if candidates is None:
            try:
                procs = len(os.sched_getaffinity(0))
            except AttributeError:
                procs = os.cpu_count() or 1
            candidates = sorted({max(1, procs // 4), max(1, procs // 2),
                                 max(1, procs - 1)})
        stream = stream or torch.cuda.current_stream(self.device)
        best, best_ms = self.threads, None
        for t in candidates:
            self.threads = int(t)
            self.run(stream)                      # settle at this count
            start = torch.cuda.Event(enable_timing=True)
            start.record(stream)
            end = None
            for _ in range(reps):
                end = self.run(stream)
            end.synchronize()
            ms = start.elapsed_time(end) / reps
            if best_ms is None or ms < best_ms:
                best, best_ms = int(t), ms
        self.threads = best
        return best

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
