"""Exact dual regional-extrema masks on B200 (sm_100a) -- Python host mirror.

The compute path is ``libsparseseam.so`` (hand-written CUDA, C ABI declared in
``include/sparse_seam.h``).  This module binds that ABI with ctypes and uses
PyTorch only for device memory and streams.  There is no CPU fallback: if the
library is missing, every entry point raises.

Reference-named mirror of the route's host interface (paths inside the
reference repository):
  allocate_buffers / free_buffers
      harness/primary/snapshot_sparse_seam_cuda_v1_0.cu:710-750
  run_sparse_resident   (device-resident image in, masks left on the device)
      harness/primary/gpu_common_v0_6.cu:137-206
  run_sparse_seam       (host image in, host masks out, kernel ms, fragments)
      harness/primary/snapshot_sparse_seam_cuda_v1_0.cu:753-878
As in the reference, device invariant failures surface as exceptions when the
status is read back (gpu_common_v0_6.cu:377-387).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libsparseseam.so")

TILES = (16, 32, 64)
HAS_GREATER = 1
HAS_SMALLER = 2
TOUCHES_SEAM = 4

STATUS = {
    0: "SS_OK",
    1: "SS_ERR_INVALID_VALUE",
    2: "SS_ERR_UNSUPPORTED_TILE",
    3: "SS_ERR_WORKSPACE_TOO_SMALL",
    4: "SS_ERR_MISALIGNED",
    5: "SS_ERR_TOO_LARGE",
    6: "SS_ERR_CUDA",
    7: "SS_ERR_FRAGMENT_OVERFLOW",
    8: "SS_ERR_RECORD_RANGE",
    9: "SS_ERR_INVARIANT",
    10: "SS_ERR_SPIN_LIMIT",
    11: "SS_ERR_WORKSPACE_UNINITIALIZED",
    12: "SS_ERR_HOST_ALLOC",
    13: "SS_ERR_EXCEEDS_STATIC_SCRATCH",
}


class SparseSeamError(RuntimeError):
    """A non-SS_OK status from the library."""

    def __init__(self, status: int, where: str):
        self.status = int(status)
        super().__init__(f"{where}: {STATUS.get(self.status, self.status)}")


class Stats(ctypes.Structure):
    _fields_ = [
        ("device_error", ctypes.c_uint32),
        ("error_detail", ctypes.c_uint32),
        ("active_fragments", ctypes.c_uint64),
        ("tiles", ctypes.c_uint64),
        ("flipped_tiles", ctypes.c_uint64),
        ("live_pixels", ctypes.c_uint64),
    ]


class ImageDesc(ctypes.Structure):
    _fields_ = [
        ("image", ctypes.c_void_p),
        ("maxima", ctypes.c_void_p),
        ("minima", ctypes.c_void_p),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("pitch", ctypes.c_int32),
        ("out_pitch", ctypes.c_int32),
    ]


class Launch(ctypes.Structure):
    """Per-call launch choices (ss_launch): the batch autotuner's knobs."""
    _fields_ = [
        ("warps", ctypes.c_int32),
        ("persistent", ctypes.c_int32),
        ("group", ctypes.c_int32),
        ("passes", ctypes.c_int32),
        ("flatten", ctypes.c_int32),
    ]


# Serving loop (ss_server_*).
class Request(ctypes.Structure):
    _fields_ = [
        ("image", ctypes.c_void_p),
        ("maxima", ctypes.c_void_p),
        ("minima", ctypes.c_void_p),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("pitch", ctypes.c_int32),
        ("out_pitch", ctypes.c_int32),
        ("flags", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("user", ctypes.c_uint64),
    ]


class Completion(ctypes.Structure):
    _fields_ = [
        ("ticket", ctypes.c_uint64),
        ("user", ctypes.c_uint64),
        ("status", ctypes.c_int32),
        ("batch_images", ctypes.c_int32),
        ("submit_ns", ctypes.c_int64),
        ("admit_ns", ctypes.c_int64),
        ("launch_ns", ctypes.c_int64),
        ("done_ns", ctypes.c_int64),
    ]


class ServerConfig(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("tile", ctypes.c_int32),
        ("persistent", ctypes.c_int32),
        ("inflight", ctypes.c_int32),
        ("max_batch_images", ctypes.c_int32),
        ("unpack_threads", ctypes.c_int32),
        ("batch_tiles", ctypes.c_int64),
        ("pool_bytes", ctypes.c_uint64),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_uint64),
        ("completed", ctypes.c_uint64),
        ("batches", ctypes.c_uint64),
        ("pixels", ctypes.c_uint64),
        ("pool_bytes", ctypes.c_uint64),
        ("pool_high_water", ctypes.c_uint64),
        ("max_batch_images_seen", ctypes.c_uint32),
        ("inflight_high_water", ctypes.c_uint32),
    ]

    def as_dict(self) -> Dict[str, int]:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


_LIB: Optional[ctypes.CDLL] = None

# name -> (restype, argtypes); every symbol include/sparse_seam.h declares.
_VP = ctypes.c_void_p
_SZ = ctypes.c_size_t
_I = ctypes.c_int
SIGNATURES = {
    "ss_status_string": (ctypes.c_char_p, [_I]),
    "ss_abi_version": (_I, []),
    "ss_workspace_bytes": (_I, [_I, _I, _I, ctypes.POINTER(_SZ)]),
    "ss_workspace_init": (_I, [_VP, _SZ, _VP]),
    "ss_extrema": (_I, [_VP, _I, _I, _I, _I, _VP, _VP, _I, _VP, _SZ, _VP]),
    "ss_read_status": (_I, [_VP, _SZ, _VP, ctypes.POINTER(Stats)]),
    "ss_context_create": (_I, [_I, ctypes.POINTER(_VP)]),
    "ss_context_destroy": (None, [_VP]),
    "ss_extrema_host": (_I, [_VP, _VP, _I, _I, _I, _I, _VP, _VP, _I,
                             ctypes.POINTER(ctypes.c_float),
                             ctypes.POINTER(ctypes.c_uint64)]),
    "ss_batch_plan_bytes": (_I, [_I, ctypes.c_int64, ctypes.POINTER(_SZ)]),
    "ss_batch_tiles": (_I, [ctypes.POINTER(ImageDesc), _I, _I,
                            ctypes.POINTER(ctypes.c_int64)]),
    "ss_batch_plan_fill": (_I, [ctypes.POINTER(ImageDesc), _I, _I, _VP, _SZ,
                                ctypes.POINTER(_SZ)]),
    "ss_extrema_batch": (_I, [_VP, _VP, _SZ, _I, _VP, _SZ, _VP]),
    "ss_extrema_batch_pass": (_I, [_VP, _VP, _SZ, _I, _I, _VP, _SZ, _VP]),
    "ss_set_kernel_config": (_I, [_I, _I]),
    "ss_get_kernel_config": (_I, [_I, ctypes.POINTER(_I)]),
    "ss_empty_launches": (_I, [_I, _I, _I, _VP]),
    "ss_extrema_static_scratch": (_I, [_VP, _I, _I, _I, _I, _VP, _VP, _I,
                                       _VP]),
    "ss_static_scratch_read_status": (_I, [_VP, ctypes.POINTER(Stats)]),
    "ss_extrema_batch_launch": (_I, [_VP, _VP, _SZ, ctypes.POINTER(Launch),
                                     _VP, _SZ, _VP]),
    "ss_server_create": (_I, [ctypes.POINTER(ServerConfig),
                              ctypes.POINTER(_VP)]),
    "ss_server_submit": (_I, [_VP, ctypes.POINTER(Request),
                              ctypes.POINTER(ctypes.c_uint64)]),
    "ss_server_poll": (_I, [_VP, ctypes.POINTER(Completion), _I,
                            ctypes.POINTER(_I), _I]),
    "ss_server_get_stats": (_I, [_VP, ctypes.POINTER(ServerStats)]),
    "ss_server_destroy": (None, [_VP]),
    "ss_pack_masks": (_I, [_VP, _VP, ctypes.c_uint64, _VP, _VP, _VP]),
    "ss_unpack_masks": (_I, [_VP, _VP, ctypes.c_uint64, _VP, _VP, _I]),
    "ss_enqueue_unpack_masks": (_I, [_VP, _VP, ctypes.c_uint64, _VP, _VP, _I,
                                     _VP]),
    "ss_extrema_levels": (_I, [_VP, _I, _I, _I, _I, _I, _VP, _VP, _I, _VP,
                               _SZ, _VP]),
    "ss_batch_plan_set_levels": (_I, [_VP, _SZ, _I, _I]),
    "ss_read_image": (_I, [ctypes.c_char_p, _VP, _SZ, ctypes.POINTER(_I),
                           ctypes.POINTER(_I)]),
    "ss_write_pgm": (_I, [ctypes.c_char_p, _VP, _I, _I, _I]),
}


def read_image(path: str) -> np.ndarray:
    """An image file (PGM, PNG, BMP, JPEG or TIFF) as a 2-D uint8 array, 8-bit gray as the
    reference's cv::imread(path, IMREAD_GRAYSCALE) reads it."""
    w, h = _I(0), _I(0)
    p = os.fsencode(path)
    _check(lib().ss_read_image(p, None, 0, ctypes.byref(w), ctypes.byref(h)),
           f"ss_read_image({path})")
    out = np.empty((h.value, w.value), dtype=np.uint8)
    _check(lib().ss_read_image(p, out.ctypes.data, out.size, ctypes.byref(w),
                               ctypes.byref(h)), f"ss_read_image({path})")
    return out


def write_pgm(path: str, image: np.ndarray) -> None:
    """Writes a 2-D uint8 array as a binary PGM."""
    image = np.ascontiguousarray(image, dtype=np.uint8)
    _check(lib().ss_write_pgm(os.fsencode(path), image.ctypes.data,
                              image.shape[1], image.shape[0], image.shape[1]),
           f"ss_write_pgm({path})")


def lib() -> ctypes.CDLL:
    """Loads the CUDA route library; raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBRARY):
            raise RuntimeError(
                f"{LIBRARY} is missing: build it with "
                "`python sparse-seam_b200/build.py` (there is no CPU fallback)")
        handle = ctypes.CDLL(LIBRARY)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = handle
    return _LIB


def _check(status: int, where: str) -> None:
    if status != 0:
        raise SparseSeamError(status, where)


def _stream_handle(stream) -> int:
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    return int(stream.cuda_stream)


def set_kernel_config(tile: int, warps: int) -> None:
    """Selects the kernels used for `tile` (see ss_set_kernel_config)."""
    _check(lib().ss_set_kernel_config(tile, warps), "ss_set_kernel_config")


def get_kernel_config(tile: int) -> int:
    out = ctypes.c_int(0)
    _check(lib().ss_get_kernel_config(tile, ctypes.byref(out)),
           "ss_get_kernel_config")
    return int(out.value)


KERNEL_CONFIGS = {16: (4, 2, 8), 32: (-4, -2, 4, 8, 16), 64: (-4, 8, 16)}


def workspace_bytes(width: int, height: int, tile: int = 32) -> int:
    out = ctypes.c_size_t(0)
    _check(lib().ss_workspace_bytes(width, height, tile, ctypes.byref(out)),
           "ss_workspace_bytes")
    return int(out.value)


class Workspace:
    """Device workspace (a torch uint8 buffer, 256-byte aligned), initialised."""

    def __init__(self, nbytes: int, device=None, stream=None):
        import torch
        self.nbytes = int(nbytes)
        self.buffer = torch.empty(self.nbytes + 256, dtype=torch.uint8,
                                  device=device or "cuda")
        base = self.buffer.data_ptr()
        self.offset = (-base) % 256
        self.ptr = base + self.offset
        self.init(stream)

    @classmethod
    def for_image(cls, width: int, height: int, tile: int = 32, **kw):
        return cls(workspace_bytes(width, height, tile), **kw)

    def init(self, stream=None) -> None:
        """Resets the workspace and waits for the reset, so the workspace is
        ready for work enqueued on any stream afterwards."""
        import torch
        st = stream or torch.cuda.current_stream(self.buffer.device)
        _check(lib().ss_workspace_init(self.ptr, self.nbytes,
                                       _stream_handle(st)),
               "ss_workspace_init")
        st.synchronize()

    def read_status(self, stream=None, raise_on_error: bool = True) -> Stats:
        stats = Stats()
        st = lib().ss_read_status(self.ptr, self.nbytes,
                                  _stream_handle(stream), ctypes.byref(stats))
        if st != 0 and raise_on_error:
            raise SparseSeamError(st, f"device (detail {stats.error_detail})")
        return stats


def _check_image_tensor(image):
    import torch
    if image.dtype != torch.uint8 or image.dim() != 2 or not image.is_cuda:
        raise ValueError("image must be a 2-D uint8 CUDA tensor")
    if image.stride(1) != 1:
        raise ValueError("image rows must be contiguous (stride(1) == 1)")
    return image.shape[0], image.shape[1], image.stride(0)


def extrema(image, tile: int = 32, maxima=None, minima=None,
            workspace: Optional[Workspace] = None, stream=None,
            check: bool = False, levels: int = 0):
    """Regional maxima / minima masks of a device image (uint8, H x W).

    Enqueues the route on `stream` (torch's current stream by default) and
    returns (maxima, minima) as uint8 CUDA tensors with 0/255 values.  With
    check=True the stream is synchronised and device errors raise.  With
    `levels` (2..256) the masks are those of the image re-quantised to that
    many gray levels, done inside the tile load (ss_extrema_levels).
    """
    import torch
    h, w, pitch = _check_image_tensor(image)
    if maxima is None:
        maxima = torch.empty((h, w), dtype=torch.uint8, device=image.device)
    if minima is None:
        minima = torch.empty((h, w), dtype=torch.uint8, device=image.device)
    for m in (maxima, minima):
        if m.shape != (h, w) or m.dtype != torch.uint8 or m.stride(1) != 1:
            raise ValueError("output masks must be uint8 H x W, rows contiguous")
    if maxima.stride(0) != minima.stride(0):
        raise ValueError("both masks must share one row pitch")
    if workspace is None:
        workspace = Workspace.for_image(w, h, tile, device=image.device,
                                        stream=stream)
    if levels:
        st = lib().ss_extrema_levels(image.data_ptr(), w, h, pitch, tile,
                                     int(levels), maxima.data_ptr(),
                                     minima.data_ptr(), maxima.stride(0),
                                     workspace.ptr, workspace.nbytes,
                                     _stream_handle(stream))
        _check(st, "ss_extrema_levels")
    else:
        st = lib().ss_extrema(image.data_ptr(), w, h, pitch, tile,
                              maxima.data_ptr(), minima.data_ptr(),
                              maxima.stride(0), workspace.ptr,
                              workspace.nbytes, _stream_handle(stream))
        _check(st, "ss_extrema")
    if check:
        workspace.read_status(stream)
    return maxima, minima


class BatchPlan:
    """Many device images of uneven sizes, run by one launch pair.

    `images`, `maxima`, `minima` are lists of uint8 CUDA tensors (H_i x W_i).
    The plan (image table + tile-to-image map) is built on the host by the
    library and copied to the device once; it can be replayed, including
    inside a captured CUDA graph, for as long as the tensors live.
    """

    def __init__(self, images: Sequence, maxima: Sequence, minima: Sequence,
                 tile: int = 32, stream=None, levels=None):
        import torch
        if not (len(images) == len(maxima) == len(minima)):
            raise ValueError("images / maxima / minima lengths differ")
        self.tile = tile
        self.images, self.maxima, self.minima = list(images), list(maxima), \
            list(minima)
        n = len(images)
        descs = (ImageDesc * max(n, 1))()
        for i, (im, mx, mn) in enumerate(zip(images, maxima, minima)):
            h, w, pitch = _check_image_tensor(im)
            if mx.shape != (h, w) or mn.shape != (h, w) or \
                    mx.stride(0) != mn.stride(0):
                raise ValueError(f"image {i}: mask shape / pitch mismatch")
            descs[i] = ImageDesc(im.data_ptr(), mx.data_ptr(), mn.data_ptr(),
                                 w, h, pitch, mx.stride(0))
        self._descs = descs
        self.count = n
        tiles = ctypes.c_int64(0)
        _check(lib().ss_batch_tiles(descs, n, tile, ctypes.byref(tiles)),
               "ss_batch_tiles")
        self.total_tiles = int(tiles.value)
        nbytes = ctypes.c_size_t(0)
        _check(lib().ss_batch_plan_bytes(n, self.total_tiles,
                                         ctypes.byref(nbytes)),
               "ss_batch_plan_bytes")
        self.plan_bytes = int(nbytes.value)
        self.host_plan = np.zeros(self.plan_bytes, dtype=np.uint8)
        ws = ctypes.c_size_t(0)
        _check(lib().ss_batch_plan_fill(
            descs, n, tile, self.host_plan.ctypes.data, self.plan_bytes,
            ctypes.byref(ws)), "ss_batch_plan_fill")
        self.workspace_bytes = int(ws.value)
        if levels is not None:
            # One gray-level count for all images, or one per image.
            per = list(levels) if hasattr(levels, "__len__") else [levels] * n
            if len(per) != n:
                raise ValueError("one levels value per image")
            for i, lv in enumerate(per):
                _check(lib().ss_batch_plan_set_levels(
                    self.host_plan.ctypes.data, self.plan_bytes, i, int(lv)),
                    "ss_batch_plan_set_levels")
        device = images[0].device if n else "cuda"
        self._dev = torch.empty(self.plan_bytes + 256, dtype=torch.uint8,
                                device=device)
        off = (-self._dev.data_ptr()) % 256
        self.device_plan = self._dev[off:off + self.plan_bytes]
        self.device_plan.copy_(torch.from_numpy(self.host_plan))
        if stream is not None:
            stream.wait_stream(torch.cuda.current_stream())

    def make_workspace(self, stream=None) -> Workspace:
        return Workspace(self.workspace_bytes, device=self._dev.device,
                         stream=stream)

    def run(self, workspace: Workspace, persistent: bool = False,
            stream=None) -> None:
        st = lib().ss_extrema_batch(
            self.host_plan.ctypes.data, self.device_plan.data_ptr(),
            self.plan_bytes, 1 if persistent else 0, workspace.ptr,
            workspace.nbytes, _stream_handle(stream))
        _check(st, "ss_extrema_batch")

    def run_launch(self, workspace: Workspace, warps: int = 0,
                   persistent: bool = False, group: int = 0, passes: int = 0,
                   flatten: int = 0, stream=None) -> None:
        """ss_extrema_batch_launch: explicit kernel family (0 = the tile's
        default), schedule, seam/resolve tiles per warp (0 = automatic),
        passes (0 = all) and fragment flatten schedule (0 halving, 1
        compress in the flags pass, 2 separate compress pass)."""
        launch = Launch(int(warps), 1 if persistent else 0, int(group),
                        int(passes), int(flatten))
        st = lib().ss_extrema_batch_launch(
            self.host_plan.ctypes.data, self.device_plan.data_ptr(),
            self.plan_bytes, ctypes.byref(launch), workspace.ptr,
            workspace.nbytes, _stream_handle(stream))
        _check(st, "ss_extrema_batch_launch")

    def run_pass(self, workspace: Workspace, which: int,
                 persistent: bool = False, stream=None) -> None:
        """One pass of the split form, enqueued in the order 1, 4, 2:
        1 = tile pass, 4 = seam pass, 2 = resolve pass."""
        st = lib().ss_extrema_batch_pass(
            self.host_plan.ctypes.data, self.device_plan.data_ptr(),
            self.plan_bytes, 1 if persistent else 0, which, workspace.ptr,
            workspace.nbytes, _stream_handle(stream))
        _check(st, "ss_extrema_batch_pass")


def extrema_batch(images: Sequence, tile: int = 32, persistent: bool = False,
                  stream=None, check: bool = True) -> Tuple[List, List]:
    """One-shot batch: allocates outputs, plan and workspace, runs, returns."""
    import torch
    maxima = [torch.empty_like(im) for im in images]
    minima = [torch.empty_like(im) for im in images]
    plan = BatchPlan(images, maxima, minima, tile=tile, stream=stream)
    ws = plan.make_workspace(stream=stream)
    plan.run(ws, persistent=persistent, stream=stream)
    if check:
        ws.read_status(stream)
    return maxima, minima


# ---------------------------------------------------------------------------
# Reference-named mirror
# ---------------------------------------------------------------------------

@dataclass
class SparseDeviceBuffers:
    """Device buffers of one image size (the reference's DeviceBuffers)."""
    image: object
    maxima: object
    minima: object
    workspace: Workspace
    tile: int
    width: int
    height: int


def allocate_buffers(width: int, height: int, tile: int = 32,
                     device="cuda") -> SparseDeviceBuffers:
    import torch
    mk = lambda: torch.empty((height, width), dtype=torch.uint8,  # noqa: E731
                             device=device)
    return SparseDeviceBuffers(mk(), mk(), mk(),
                               Workspace.for_image(width, height, tile,
                                                   device=device),
                               tile, width, height)


def free_buffers(buffers: SparseDeviceBuffers) -> None:
    buffers.image = buffers.maxima = buffers.minima = None
    buffers.workspace = None


def run_sparse_resident(buffers: SparseDeviceBuffers, width: int,
                        height: int, stream=None) -> int:
    """Enqueues the route on the image already in buffers.image; returns 1."""
    if (width, height) != (buffers.width, buffers.height):
        raise ValueError("buffers were allocated for another size")
    extrema(buffers.image, buffers.tile, buffers.maxima, buffers.minima,
            buffers.workspace, stream=stream)
    return 1


def run_sparse_seam(buffers: SparseDeviceBuffers, image: np.ndarray,
                    stream=None):
    """Host image in; returns (kernel_ms, maxima, minima, active_fragments)."""
    import torch
    h, w = image.shape
    if (w, h) != (buffers.width, buffers.height):
        raise ValueError("buffers were allocated for another size")
    st = stream or torch.cuda.current_stream()
    buffers.image.copy_(torch.from_numpy(np.ascontiguousarray(image)),
                        non_blocking=False)
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(st)
    run_sparse_resident(buffers, w, h, stream=st)
    stop.record(st)
    stats = buffers.workspace.read_status(st)
    maxima = buffers.maxima.cpu().numpy()
    minima = buffers.minima.cpu().numpy()
    return start.elapsed_time(stop), maxima, minima, int(stats.active_fragments)
