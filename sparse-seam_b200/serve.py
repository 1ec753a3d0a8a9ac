"""Serving: the library's continuous-batching request loop (ss_server_*).

A `Server` owns a device pool for request buffers and a few batch slots; its
native worker thread admits requests by HBM footprint, batches whatever has
arrived whenever a slot frees, overlaps batches on the device and copies the
masks back.  `poisson_trace` and `run_trace` drive it with an open-loop
arrival process and report latency percentiles and throughput.

Timestamps are CLOCK_MONOTONIC nanoseconds on both sides (the library's
clock_gettime and Python's time.monotonic_ns), so a request's latency is its
completion time minus its scheduled arrival, whatever delay the submitting
thread had.
"""
from __future__ import annotations

import ctypes
import importlib
import os
import time
from dataclasses import dataclass
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

_pkg = importlib.import_module(__package__)

REQUEST_DEVICE = 1
Request = _pkg.Request
Completion = _pkg.Completion
ServerConfig = _pkg.ServerConfig
ServerStats = _pkg.ServerStats


def _ptr(t) -> int:
    return t.data_ptr() if hasattr(t, "data_ptr") else t.ctypes.data


def _pitch(t) -> int:
    return int(t.stride(0)) if hasattr(t, "stride") and callable(t.stride) \
        else int(t.strides[0])


class Server:
    """A running serving loop; close() (or a with-block) finishes every
    submitted request and frees the device memory."""

    def __init__(self, tile: int = 32, persistent: bool = True,
                 inflight: int = 2, max_batch_images: int = 512,
                 batch_tiles: int = 1 << 16, pool_bytes: int = 1 << 30,
                 device: int = 0, unpack_threads: int = 0):
        self.config = ServerConfig(device, tile, 1 if persistent else 0,
                                   inflight, max_batch_images,
                                   unpack_threads, batch_tiles, pool_bytes)
        handle = ctypes.c_void_p()
        _pkg._check(_pkg.lib().ss_server_create(ctypes.byref(self.config),
                                                ctypes.byref(handle)),
                    "ss_server_create")
        self._h = handle
        self._buf = (Completion * 1024)()
        self._keep: Dict[int, tuple] = {}

    def submit(self, image, maxima, minima, device: bool = False,
               user: int = 0) -> int:
        """Queues one image.  Host tensors / arrays should be pinned for the
        copies to overlap; with device=True all three are CUDA tensors."""
        h, w = int(image.shape[0]), int(image.shape[1])
        req = Request(_ptr(image), _ptr(maxima), _ptr(minima), w, h,
                      _pitch(image), _pitch(maxima),
                      REQUEST_DEVICE if device else 0, 0, int(user))
        ticket = ctypes.c_uint64(0)
        _pkg._check(_pkg.lib().ss_server_submit(self._h, ctypes.byref(req),
                                                ctypes.byref(ticket)),
                    "ss_server_submit")
        self._keep[int(ticket.value)] = (image, maxima, minima)
        return int(ticket.value)

    def submit_file(self, path: str, user: int = 0):
        """Decodes an image file (PGM, PNG, BMP, JPEG or TIFF, read as the
        reference's cv::imread(path, IMREAD_GRAYSCALE) reads it) straight
        into pinned host memory and queues it.  Returns (ticket, maxima,
        minima): the masks arrive in the returned pinned buffers when the
        request's completion is polled."""
        import torch
        w, h = ctypes.c_int(0), ctypes.c_int(0)
        p = os.fsencode(path)
        _pkg._check(_pkg.lib().ss_read_image(p, None, 0, ctypes.byref(w),
                                             ctypes.byref(h)),
                    f"ss_read_image({path})")
        shape = (h.value, w.value)
        pin = dict(dtype=torch.uint8, pin_memory=True)
        image = torch.empty(shape, **pin)
        _pkg._check(_pkg.lib().ss_read_image(p, image.data_ptr(),
                                             image.numel(), ctypes.byref(w),
                                             ctypes.byref(h)),
                    f"ss_read_image({path})")
        maxima = torch.empty(shape, **pin)
        minima = torch.empty(shape, **pin)
        return self.submit(image, maxima, minima, user=user), maxima, minima

    def poll(self, timeout_us: int = 0) -> List[Completion]:
        n = ctypes.c_int(0)
        _pkg._check(_pkg.lib().ss_server_poll(self._h, self._buf,
                                              len(self._buf), ctypes.byref(n),
                                              int(timeout_us)),
                    "ss_server_poll")
        out = []
        for i in range(n.value):
            c = Completion.from_buffer_copy(self._buf[i])
            self._keep.pop(int(c.ticket), None)
            out.append(c)
        return out

    def stats(self) -> Dict[str, int]:
        s = ServerStats()
        _pkg._check(_pkg.lib().ss_server_get_stats(self._h, ctypes.byref(s)),
                    "ss_server_get_stats")
        return s.as_dict()

    def close(self) -> None:
        if self._h:
            _pkg.lib().ss_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Open-loop load
# ---------------------------------------------------------------------------

def serve_files(server: Server, paths: Sequence[str],
                timeout_s: float = 600.0) -> Dict[str, Tuple]:
    """Serves image files: each is decoded into pinned memory and queued as
    soon as it is read (decoding the next file overlaps the GPU work of the
    earlier ones).  Returns {path: (maxima, minima)}; raises on a failed
    request."""
    pending = {}
    for i, path in enumerate(paths):
        ticket, mx, mn = server.submit_file(path, user=i)
        pending[ticket] = (path, mx, mn)
    out = {}
    deadline = time.monotonic() + timeout_s
    while len(out) < len(paths):
        if time.monotonic() > deadline:
            raise TimeoutError("requests did not complete in time")
        for c in server.poll(timeout_us=10_000):
            path, mx, mn = pending[int(c.ticket)]
            if c.status != 0:
                raise _pkg.SparseSeamError(int(c.status),
                                           f"served request {path}")
            out[path] = (mx, mn)
    return out


def poisson_trace(rate: float, duration_s: float, seed: int = 0) -> np.ndarray:
    """Arrival offsets in nanoseconds of a Poisson process."""
    rng = np.random.default_rng(seed)
    n = max(1, int(rate * duration_s * 1.2) + 16)
    gaps = rng.exponential(1.0 / rate, size=n)
    t = np.cumsum(gaps)
    return (t[t < duration_s] * 1e9).astype(np.int64)


@dataclass
class TraceResult:
    requests: int
    pixels: int
    p50_ms: float
    p90_ms: float
    p99_ms: float
    max_ms: float
    makespan_s: float
    gpix_s: float
    failures: int
    mean_batch_images: float
    stats: Dict[str, int]

    def as_dict(self) -> Dict:
        return {k: (round(v, 4) if isinstance(v, float) else v)
                for k, v in self.__dict__.items()}


def run_trace(server: Server, arrivals_ns: Sequence[int],
              make_request: Callable[[int], Tuple], device: bool = False,
              poll_us: int = 200) -> TraceResult:
    """Submits request i at start + arrivals_ns[i] (open loop), collects every
    completion, and reports latency (completion - scheduled arrival)."""
    n = len(arrivals_ns)
    planned = {}
    pixels = {}
    done: List[Completion] = []
    start = time.monotonic_ns() + 2_000_000
    i = 0
    while i < n:
        now = time.monotonic_ns()
        due = start + int(arrivals_ns[i])
        if now >= due:
            image, mx, mn = make_request(i)
            t = server.submit(image, mx, mn, device=device, user=i)
            planned[t] = due
            pixels[t] = int(image.shape[0]) * int(image.shape[1])
            i += 1
            continue
        wait_us = (due - now) // 1000
        if wait_us > 2 * poll_us:
            done.extend(server.poll(timeout_us=poll_us))
        elif wait_us > 50:
            done.extend(server.poll(timeout_us=0))
    while len(done) < n:
        done.extend(server.poll(timeout_us=10_000))
    lat = np.array([(c.done_ns - planned[int(c.ticket)]) / 1e6 for c in done])
    first = start + int(arrivals_ns[0]) if n else start
    last = max(c.done_ns for c in done) if done else first
    total_px = sum(pixels.values())
    span = max(1e-9, (last - first) / 1e9)
    return TraceResult(
        requests=n, pixels=total_px,
        p50_ms=float(np.percentile(lat, 50)) if n else 0.0,
        p90_ms=float(np.percentile(lat, 90)) if n else 0.0,
        p99_ms=float(np.percentile(lat, 99)) if n else 0.0,
        max_ms=float(lat.max()) if n else 0.0,
        makespan_s=span, gpix_s=total_px / span / 1e9,
        failures=sum(1 for c in done if c.status != 0),
        mean_batch_images=float(np.mean([c.batch_images for c in done]))
        if n else 0.0,
        stats=server.stats())
