#!/usr/bin/env python
"""Benchmark: exact dual regional-extrema masks (bit-exact), Gpix/s.

Workload (one "step"): the natural-image-like corpus -- 100 images of
2040x1356 plus 100 of 481x321 uint8 smooth noise (sigma 1/4/16 px fields,
weights 0.2/0.3/0.5, U{-2..2} jitter), tile T = 32, all 256 gray levels.
292.5 Mpix per step; inputs (292 MB) plus masks (585 MB) exceed the 126 MB
L2, so no L2 flush is needed between steps.

  value        whole-job Gpix/s of the batched form: both passes of the route
               over the whole corpus in one launch pair, replayed from a CUDA
               graph, inputs already resident in HBM, timed with CUDA events
               (max over ranks)
  e2e          the same metric through the public host-to-host API (pinned
               host images -> device -> both masks back to pinned host
               memory, chunked so copies overlap the kernels)
  per_image    the plain per-image launch (one ss_extrema per image, graph
               replayed) -- the form the batched path must beat
  roofline     the tile pass (dominant kernel) against the 3 B/pixel
               compulsory traffic (1 B read + 2 B written) at the measured
               HBM copy bandwidth
  cpu_baseline the CPU union-find oracle over the same corpus on the host's
               cores (one image per thread)
  reference_gpu  the reference's own Sparse-Seam v1.0 and Global-UF routes,
               compiled unchanged for sm_100a, per-image protocol of the
               reference harness (median of reps), on a sample of the corpus

--impl reference times the CPU exact path (the reference has no CPU
implementation of this route; the oracle port stands in) on the same corpus.

Multi-GPU: one process per GPU (torchrun); every rank processes its own
corpus (replicas, weak scaling); no collective touches the data path.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Gpix/s dual masks (bit-exact), batched vs per-image; p50/p99 served latency"
UNIT = "Gpix/s"
BYTES_PER_PIXEL = 3  # 1 B image read + 2 B mask writes


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="sparse-seam-b200",
                   choices=["sparse-seam-b200", "reference"])
    p.add_argument("--tile", type=int, default=32)
    p.add_argument("--warps", type=int, default=0,
                   help="kernel family for --tile (ss_set_kernel_config: "
                        "< 0 row-scan, > 0 CTA-per-tile warps; 0 = the "
                        "library's default)")
    p.add_argument("--large", type=int, default=100)
    p.add_argument("--small", type=int, default=100)
    p.add_argument("--quick", action="store_true",
                   help="skip the secondary measurements (per-image, e2e, "
                        "CPU baseline, reference GPU routes)")
    p.add_argument("--no-extra", action="store_true",
                   help="skip the uneven-size batch, serving and resolution "
                        "sections")
    p.add_argument("--passes-only", action="store_true",
                   help="only run the split-pass loop (for profiling)")
    p.add_argument("--host-only", action="store_true",
                   help="only run the host-to-host form (pack kernel and "
                        "host expansion; for profiling)")
    p.add_argument("--levels", type=int, default=256,
                   help="re-quantise the corpus to this many gray levels")
    p.add_argument("--sweep", action="store_true",
                   help="add the quantisation x tile sweep of the corpus")
    p.add_argument("--schedule", default="auto",
                   choices=["auto", "grid", "persistent"],
                   help="tile-pass schedule of the timed steps: the faster "
                        "of the two in a short probe (default), or pinned "
                        "(for profiling, where the probe's timings are the "
                        "profiler's)")
    p.add_argument("--serve-seconds", type=float, default=60.0,
                   help="duration of each Poisson rate of the served stream")
    return p.parse_args()


# ---------------------------------------------------------------------------
# Distributed plumbing (one process per GPU)
# ---------------------------------------------------------------------------

class Dist:
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE).

    Only timing crosses ranks (a barrier and a max over the measured times);
    the images are independent, so no collective touches the data path.
    `backend` is "nccl" on GPUs; the CPU tests use "gloo".
    """

    def __init__(self, backend: str = "nccl"):
        import torch
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.pg = False
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            kwargs = {}
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                kwargs["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(
                backend, timeout=datetime.timedelta(seconds=300), **kwargs)
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch
            import torch.distributed as dist
            if self.backend == "nccl":
                dist.barrier(device_ids=[self.local])
                torch.cuda.synchronize()
            else:
                dist.barrier()

    def max(self, value: float) -> float:
        if not self.pg:
            return value
        import torch
        import torch.distributed as dist
        device = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([value], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Clock sampling during the timed region
# ---------------------------------------------------------------------------

REASONS = [
    ("hw_slowdown", "clocks_event_reasons.hw_slowdown"),
    ("hw_thermal_slowdown", "clocks_event_reasons.hw_thermal_slowdown"),
    ("sw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown"),
    ("sw_power_cap", "clocks_event_reasons.sw_power_cap"),
]


class ClockSampler:
    """SM clock, power and throttle reasons sampled during a timed region.

    NVML (read-only queries) is polled every ~2 ms on a thread, and only the
    samples taken between mark_start() and mark_end() count, so even a timed
    region of a few milliseconds gets samples of its own.  Without NVML,
    `nvidia-smi -lms 10` is read instead (coarser).  Nothing is changed on
    the GPU.
    """

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.samples = []          # (t, sm_mhz, max_mhz, power_w, reasons)
        self._stop = threading.Event()
        self._thread = None
        self._proc = None
        self.window = (None, None)
        self.source = None

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            handle = None
            try:
                # The CUDA device by UUID (NVML numbers every GPU of the
                # host, whatever CUDA_VISIBLE_DEVICES selects).
                import torch
                uuid = str(torch.cuda.get_device_properties(
                    self.device_index).uuid)
                handle = pynvml.nvmlDeviceGetHandleByUUID(
                    uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except Exception:
                handle = pynvml.nvmlDeviceGetHandleByIndex(self.device_index)
            bits = {
                "hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown":
                    pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown":
                    pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap,
            }
            max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(
                handle, pynvml.NVML_CLOCK_SM)

            def poll():
                while not self._stop.is_set():
                    t = time.monotonic()
                    try:
                        sm = pynvml.nvmlDeviceGetClockInfo(
                            handle, pynvml.NVML_CLOCK_SM)
                        pw = pynvml.nvmlDeviceGetPowerUsage(handle) / 1000.0
                        rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(
                            handle)
                    except Exception:
                        break
                    active = [n for n, b in bits.items() if rs & b]
                    self.samples.append((t, sm, max_mhz, pw, active))
                    time.sleep(0.002)
            self.source = "nvml"
            self._thread = threading.Thread(target=poll, daemon=True)
            self._thread.start()
            return
        except Exception:
            pass
        fields = ["clocks.sm", "clocks.max.sm", "power.draw"] + \
            [q for _, q in REASONS]
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={','.join(fields)}",
                 "--format=csv,noheader,nounits", "-lms", "10",
                 "-i", str(self.device_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self._proc = None
            return
        self.source = "nvidia-smi"

        def read():
            for line in self._proc.stdout:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 3 + len(REASONS):
                    continue
                try:
                    sm, mx, pw = (float(parts[0]), float(parts[1]),
                                  float(parts[2]))
                except ValueError:
                    continue
                active = [n for (n, _), v in zip(REASONS, parts[3:])
                          if v.lower().startswith("active")]
                self.samples.append((time.monotonic(), sm, mx, pw, active))
        self._thread = threading.Thread(target=read, daemon=True)
        self._thread.start()
        time.sleep(0.3)

    def mark_start(self):
        self.window = (time.monotonic(), None)

    def mark_end(self):
        self.window = (self.window[0], time.monotonic())

    def stop(self) -> dict:
        self._stop.set()
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
        if self._thread:
            self._thread.join(timeout=2)
        if self.source is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [],
                    "note": "neither NVML nor nvidia-smi available"}
        t0, t1 = self.window
        inside = [x for x in self.samples
                  if (t0 is None or x[0] >= t0) and (t1 is None or x[0] <= t1)]
        if not inside:
            inside = self.samples[-1:]
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [],
                    "samples": 0, "source": self.source}
        active = sorted({r for x in inside for r in x[4]})
        return {"sm_mhz": statistics.median(x[1] for x in inside),
                "sm_max_mhz": max(x[2] for x in inside),
                "power_w_max": max(x[3] for x in inside),
                "reasons": active, "samples": len(inside),
                "source": self.source}


# ---------------------------------------------------------------------------
# Workload
# ---------------------------------------------------------------------------

def corpus_shapes(n_large: int, n_small: int):
    return [(1356, 2040)] * n_large + [(321, 481)] * n_small


def corpus_seed_base(rank: int) -> int:
    """Each rank (replica) processes its own corpus."""
    return 7919 * rank


def make_corpus(n_large: int, n_small: int, seed_base: int, device,
                levels: int = 256):
    from importlib import import_module
    synth = import_module("sparse-seam_b200.synth")
    out = [synth.smooth_noise(h, w, seed_base + i, device=device)
           for i, (h, w) in enumerate(corpus_shapes(n_large, n_small))]
    if levels < 256:
        out = [quantize_tensor(t, levels) for t in out]
    return out


def quantize_tensor(t, levels: int):
    """The reference's re-quantisation rule on a device tensor
    (harness/quantization_and_scaling/gpu_common_quant_v0_7.cu:479-494)."""
    import torch
    b = (t.to(torch.int32) * levels) >> 8
    return ((b * 255 + (levels - 1) // 2) // (levels - 1)).to(torch.uint8)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            data = json.load(f)
        return float(data["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def committed_traffic():
    """DRAM bytes per pixel of the tile pass from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "tile_pass_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# CPU exact path (reference arm and cpu_baseline)
# ---------------------------------------------------------------------------

def time_cpu_oracle(host_images, threads: int, reps: int = 1):
    import oracle
    pixels = sum(im.size for im in host_images)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        oracle.extrema_batch(host_images, threads=threads)
        times.append(time.perf_counter() - t0)
    return pixels, times


def run_reference_arm(args, dist: Dist):
    import torch
    if dist.rank != 0:
        return 0
    device = "cuda" if torch.cuda.is_available() else "cpu"
    images = [t.cpu().numpy() for t in
              make_corpus(args.large, args.small, 0, device, args.levels)]
    threads = cpu_threads()
    pixels, _ = time_cpu_oracle(images, threads, reps=max(1, args.warmup))
    _, times = time_cpu_oracle(images, threads, reps=args.steps)
    total = sum(times)
    value = pixels * args.steps / total / 1e9
    sample = (f"the full corpus per step ({args.large} x 2040x1356 + "
              f"{args.small} x 481x321, {pixels} px), union-find oracle, "
              f"one image per thread")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 6),
        "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic (seeded smooth-noise corpus)",
        "config": config_dict(args),
        "cpu_baseline": {"value": round(value, 6), "unit": UNIT,
                         "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 6), "unit": UNIT,
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("the reference ships no CPU implementation of the route; "
                 "the C restatement of its rule (oracle/ss_oracle.c) is timed"),
    }
    print(json.dumps(line))
    return 0


def config_dict(args):
    return {
        "workload": (f"natural-image-like corpus: {args.large} x 2040x1356 + "
                     f"{args.small} x 481x321 uint8 smooth noise, "
                     f"{args.levels} levels"),
        "tile": args.tile,
        "kernel_config": args.warps or "default",
        "images_per_step": args.large + args.small,
        "pixels_per_step": sum(h * w for h, w in
                               corpus_shapes(args.large, args.small)),
        "l2": "inputs + masks (877 MB) exceed L2; no flush",
        "parallelism": f"replicas x{args.gpus}",
    }


# ---------------------------------------------------------------------------
# Reference GPU routes (checker build, oracle/_ref)
# ---------------------------------------------------------------------------

def reference_gpu_routes(host_images, tile: int, warmup=3, reps=10):
    path = os.path.join(ROOT, "oracle", "_ref", f"libssref_t{tile}.so")
    if not os.path.exists(path):
        return {"unavailable": f"{os.path.relpath(path, ROOT)} not built"}
    import numpy as np
    lib = ctypes.CDLL(path)
    u8 = ctypes.POINTER(ctypes.c_uint8)
    d = ctypes.POINTER(ctypes.c_double)
    lib.ssref_sparse_seam.argtypes = [u8, ctypes.c_int, ctypes.c_int, u8, u8,
                                      ctypes.c_int, ctypes.c_int, d, d,
                                      ctypes.POINTER(ctypes.c_longlong)]
    lib.ssref_global_uf.argtypes = [u8, ctypes.c_int, ctypes.c_int, u8, u8,
                                    ctypes.c_int, ctypes.c_int, d, d]
    out = {}
    for name in ("sparse_seam_v1_0", "global_uf"):
        pix = 0
        sec = 0.0
        h2h = 0.0
        for img in host_images:
            h, w = img.shape
            img = np.ascontiguousarray(img)
            mx = np.empty_like(img)
            mn = np.empty_like(img)
            ms = ctypes.c_double()
            hms = ctypes.c_double()
            if name == "sparse_seam_v1_0":
                frag = ctypes.c_longlong()
                rc = lib.ssref_sparse_seam(
                    img.ctypes.data_as(u8), w, h, mx.ctypes.data_as(u8),
                    mn.ctypes.data_as(u8), warmup, reps, ctypes.byref(ms),
                    ctypes.byref(hms), ctypes.byref(frag))
            else:
                rc = lib.ssref_global_uf(
                    img.ctypes.data_as(u8), w, h, mx.ctypes.data_as(u8),
                    mn.ctypes.data_as(u8), warmup, reps, ctypes.byref(ms),
                    ctypes.byref(hms))
            if rc != 0:
                out[name] = {"error": "reference route raised"}
                break
            pix += img.size
            sec += ms.value / 1e3
            h2h += hms.value / 1e3
        else:
            out[name] = {"value": round(pix / sec / 1e9, 4), "unit": UNIT,
                         "h2h_value": round(pix / h2h / 1e9, 4),
                         "protocol": (f"per image: {warmup} warm-ups, median "
                                      f"of {reps} reps; sum(px)/sum(median)")}
    out["sample"] = f"{len(host_images)} images of the corpus"
    out["tile"] = tile
    return out


# ---------------------------------------------------------------------------
# Product arm
# ---------------------------------------------------------------------------

def main():
    args = parse_args()
    import torch
    dist = Dist()
    if args.impl == "reference":
        rc = run_reference_arm(args, dist)
        dist.close()
        return rc
    from importlib import import_module
    pkg = import_module("sparse-seam_b200")
    # The served stream's plateau maps are computed by spawned worker
    # processes, started after the host-bound measurements (e2e, CPU
    # baseline), which their computation would slow.
    plateau_pool, plateau = None, None
    device = torch.device("cuda", dist.local)
    torch.cuda.set_device(device)
    tile = args.tile
    if args.warps:
        pkg.set_kernel_config(tile, args.warps)

    images = make_corpus(args.large, args.small, corpus_seed_base(dist.rank),
                         device, args.levels)
    pixels = sum(im.numel() for im in images)
    maxs = [torch.empty_like(im) for im in images]
    mins = [torch.empty_like(im) for im in images]
    plan = pkg.BatchPlan(images, maxs, mins, tile=tile)
    ws = plan.make_workspace()
    stream = torch.cuda.Stream(device)
    torch.cuda.synchronize()

    # -- correctness of this very workload (outside every timed region) ---
    plan.run(ws, persistent=False, stream=stream)
    stats = ws.read_status(stream)
    host_images = [im.cpu().numpy() for im in images]
    import numpy as np
    import oracle
    check_n = len(images) if dist.rank == 0 else 4
    idx = list(range(0, len(images), max(1, len(images) // check_n)))[:check_n]
    want_max, want_min = oracle.extrema_batch([host_images[i] for i in idx],
                                              threads=cpu_threads())
    mismatches = 0
    for j, i in enumerate(idx):
        mismatches += int((maxs[i].cpu().numpy() != want_max[j]).sum())
        mismatches += int((mins[i].cpu().numpy() != want_min[j]).sum())
    if mismatches:
        print(json.dumps({"error": "masks differ from the oracle",
                          "mismatched_pixels": mismatches}))
        return 1

    if args.passes_only:
        for _ in range(max(1, args.steps)):
            plan.run_pass(ws, 1, stream=stream)
            plan.run_pass(ws, 4, stream=stream)
            plan.run_pass(ws, 2, stream=stream)
        ws.read_status(stream)
        return 0
    if args.host_only:
        host = import_module("sparse-seam_b200.host")
        hb = host.HostBatch(host_images, tile=tile, chunks=16,
                            persistent=False, packed=True)
        for _ in range(max(1, args.steps)):
            hb.run(stream)
        stream.synchronize()
        hb.check()
        return 0

    # -- schedule: one CTA per work item vs the persistent work queue -------
    def timed(fn, reps):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(reps):
            fn()
        e.record(stream)
        e.synchronize()
        return s.elapsed_time(e) / reps

    sched = {}
    for persistent in (False, True):
        timed(lambda: plan.run(ws, persistent=persistent, stream=stream), 2)
        sched[persistent] = timed(
            lambda: plan.run(ws, persistent=persistent, stream=stream), 3)
    persistent = (sched[True] < sched[False] if args.schedule == "auto"
                  else args.schedule == "persistent")
    ws.read_status(stream)

    launches_per_run = 4 if pkg.get_kernel_config(tile) < 0 else 2

    # -- batched form, graph-replayed: the headline value ------------------
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(stream):
        plan.run(ws, persistent=persistent, stream=stream)  # warm capture path
        stream.synchronize()
        with torch.cuda.graph(graph, stream=stream):
            plan.run(ws, persistent=persistent, stream=stream)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            graph.replay()
    stream.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dist.local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    clocks.mark_start()
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for _ in range(args.steps):
            graph.replay()
        ev1.record(stream)
    ev1.synchronize()
    clocks.mark_end()
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    dist.barrier()
    ms_local = ev0.elapsed_time(ev1)
    ms_total = dist.max(ms_local)
    value = dist.world * pixels * args.steps / (ms_total / 1e3) / 1e9
    stats = ws.read_status(stream)

    # -- per-pass timing (roofline of the tile pass) ----------------------
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)]
          for _ in range(args.steps)]
    for k in range(args.steps):
        ev[k][0].record(stream)
        plan.run_pass(ws, 1, persistent=persistent, stream=stream)
        ev[k][1].record(stream)
        plan.run_pass(ws, 4, persistent=persistent, stream=stream)
        ev[k][2].record(stream)
        plan.run_pass(ws, 2, persistent=persistent, stream=stream)
        ev[k][3].record(stream)
    stream.synchronize()
    tile_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in ev)
    seam_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in ev)
    resolve_ms = statistics.mean(e[2].elapsed_time(e[3]) for e in ev)
    ws.read_status(stream)
    # Seam statistics of one step (the flip counter accumulates until read).
    plan.run(ws, persistent=persistent, stream=stream)
    step_stats = ws.read_status(stream)
    hbm, peak_kind = peaks()
    achieved = BYTES_PER_PIXEL * pixels / (tile_ms / 1e3) / 1e9
    traffic = committed_traffic()
    traffic_bytes = None
    if traffic and traffic.get("tile") == tile:
        traffic_bytes = int(traffic["dram_bytes_per_pixel"] * pixels)

    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT,
        "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_total / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic (seeded smooth-noise corpus)",
        "config": config_dict(args),
        "schedule": {"persistent": persistent, "choice": args.schedule,
                     "ms_grid": round(sched[False], 4),
                     "ms_persistent": round(sched[True], 4)},
        "gpu_launches": launches_per_run * args.steps,
        "passes_ms": {"tile_pass": round(tile_ms, 4),
                      "seam_pass": round(seam_ms, 4),
                      "resolve_pass": round(resolve_ms, 4)},
        "roofline": {"bound": "hbm", "kernel": "tile_pass_kernel",
                     "achieved": round(achieved, 2), "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4),
                     "traffic": traffic_bytes,
                     "algorithmic_bytes": BYTES_PER_PIXEL * pixels},
        "route_roofline_frac": round(
            BYTES_PER_PIXEL * pixels / (ms_total / args.steps / 1e3) / 1e9
            / hbm, 4),
        "stats": {"active_fragments": int(step_stats.active_fragments),
                  "tiles": int(step_stats.tiles),
                  "flipped_tiles_per_step": int(step_stats.flipped_tiles),
                  "live_pixels_per_step": int(step_stats.live_pixels),
                  "seam_pixel_fraction": round(
                      step_stats.live_pixels / max(1, pixels), 5)},
        "clocks": clock_info,
        "checked_images": len(idx),
        "mismatches": mismatches,
    }

    if args.sweep:
        line["sweep"] = sweep(args, pkg, images, stream)
    if not args.quick:
        line.update(secondary(args, pkg, plan, images, host_images, maxs,
                              mins, stream, dist, hbm))
        if not args.no_extra and dist.world == 1:
            # Single-GPU workloads (the uneven-size batch, the served stream
            # and the resolution sweep are defined on one B200).  The plateau
            # maps compute during the uneven-size batch.
            plateau_pool, plateau = start_plateau_maps()
            line["batched_uneven"] = uneven_section(args, pkg, device, stream)
            line["served"] = serving_section(args, pkg, device, stream,
                                             plateau)
            plateau_pool.shutdown()
            line["resolution_sweep"] = resolution_section(args, pkg, device,
                                                          stream, hbm)
    elif dist.rank == 0:
        line["cpu_baseline"] = None
        line["e2e"] = None

    line["results"] = summary(line)
    del graph
    if dist.rank == 0:
        print(json.dumps(line))
    dist.close()
    return 0


def summary(line):
    """The compact results, placed last in the JSON line (readers that keep
    only its end still see them): Gpix/s unless stated."""
    def get(*path):
        d = line
        for k in path:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return d
    out = {
        "batched": line.get("value"),
        "per_image": get("per_image", "value"),
        "single_2040x1356_us": get("single_image_2040x1356", "us_per_image"),
        "single_2040x1356": get("single_image_2040x1356", "gpix_s"),
        "launch_floor_us_1_4": [get("launch_floor_2040x1356", "us_1_launch"),
                                get("launch_floor_2040x1356", "us_4_launch")],
        "single_passes_us": line.get("single_image_passes_us"),
        "e2e": get("e2e", "value"),
        "tile_pass_frac": get("roofline", "frac"),
    }
    for t in (32, 64):
        out[f"ref_protocol_t{t}"] = {
            "product": get("ref_protocol", f"t{t}", "product", "gpix_s"),
            "sparse_seam": get("ref_protocol", f"t{t}", "reference",
                               "sparse_seam_v1_0", "value"),
            "global_uf": get("ref_protocol", f"t{t}", "reference",
                             "global_uf", "value")}
    out["uneven"] = {k: get("batched_uneven", k, "gpix_s")
                     for k in ("per_image", "batched_grid",
                               "batched_persistent", "autotuned")}
    rates = get("served", "rates_req_s") or {}
    out["served"] = {r: [v.get("p50_ms"), v.get("p99_ms"), v.get("gpix_s")]
                     for r, v in rates.items()}
    out["served_note"] = "rate: [p50 ms, p99 ms, Gpix/s]"
    out["served_duration_s"] = get("served", "duration_s")
    out["served_vs_per_image_h2h"] = [get("served", "saturated", "gpix_s"),
                                      get("served", "per_image_h2h",
                                          "gpix_s")]
    out["cpu_baseline"] = get("cpu_baseline", "value")
    out["mismatches"] = line.get("mismatches")
    return out


def sweep(args, pkg, images, stream):
    """Batched Gpix/s of the corpus re-quantised to 256/64/16/4/2 levels at
    T = 16 / 32 / 64 (the reference's quantisation and tile-size studies).
    The re-quantisation is fused into the tile load (the plan's per-image
    gray levels), so it is inside the timed region; each setting is checked
    against the oracle of the host-quantised image on two images."""
    import torch
    import oracle
    out = {}
    pixels = sum(im.numel() for im in images)
    imgs = images
    maxs = [torch.empty_like(t) for t in imgs]
    mins = [torch.empty_like(t) for t in imgs]
    for levels in (256, 64, 16, 4, 2):
        for tile in (16, 32, 64):
            plan = pkg.BatchPlan(imgs, maxs, mins, tile=tile, stream=stream,
                                 levels=levels)
            ws = plan.make_workspace(stream=stream)
            best = None
            for persistent in (False, True):
                plan.run(ws, persistent=persistent, stream=stream)
                stream.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(3):
                    plan.run(ws, persistent=persistent, stream=stream)
                e1.record(stream)
                e1.synchronize()
                ms = e0.elapsed_time(e1) / 3
                best = ms if best is None else min(best, ms)
            ws.read_status(stream)
            bad = 0
            for i in (0, len(imgs) - 1):
                h = quantize_tensor(imgs[i], levels).cpu().numpy()
                wmx, wmn = oracle.extrema(h)
                bad += int((maxs[i].cpu().numpy() != wmx).sum())
                bad += int((mins[i].cpu().numpy() != wmn).sum())
            out[f"q{levels}_t{tile}"] = {
                "gpix_s": round(pixels / (best / 1e3) / 1e9, 3),
                "ms": round(best, 4), "mismatches": bad}
            del plan, ws
    return out


def secondary(args, pkg, plan, images, host_images, maxs, mins, stream, dist,
              hbm):
    import torch
    out = {}
    tile = args.tile
    pixels = sum(im.numel() for im in images)

    # -- plain per-image launches, graph-replayed ----------------------------
    big = max(images, key=lambda t: t.numel())
    ws1 = pkg.Workspace.for_image(big.shape[1], big.shape[0], tile)

    def per_image_graph(sel):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(stream):
            for i in sel:
                pkg.extrema(images[i], tile, maxs[i], mins[i], ws1,
                            stream=stream)
            stream.synchronize()
            with torch.cuda.graph(g, stream=stream):
                for i in sel:
                    pkg.extrema(images[i], tile, maxs[i], mins[i], ws1,
                                stream=stream)
        # Warm-up replays on the timing stream, and the device drained: a
        # replay left running on another stream would fall inside the timed
        # window.
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                g.replay()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.steps):
                g.replay()
            e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        del g
        return ms

    all_ms = per_image_graph(range(len(images)))
    large = [i for i, t in enumerate(images) if t.shape == (1356, 2040)]
    large_ms = per_image_graph(large) if large else None
    ws1.read_status(stream)
    out["per_image"] = {
        "value": round(pixels / (all_ms / 1e3) / 1e9, 4), "unit": UNIT,
        "ms_per_step": round(all_ms, 4),
        "launches_per_image": 4 if pkg.get_kernel_config(tile) < 0 else 2,
    }
    if large_ms:
        px = 2040 * 1356
        per = large_ms / len(large)
        out["single_image_2040x1356"] = {
            "us_per_image": round(per * 1e3, 3),
            "gpix_s": round(px / (per / 1e3) / 1e9, 4),
            "roofline_frac": round(BYTES_PER_PIXEL * px / (per / 1e3) / 1e9
                                   / hbm, 4),
            "protocol": ("graph of one ss_extrema per image over the "
                         f"{len(large)} distinct 2040x1356 images, replayed "
                         "back to back"),
        }

    # -- e2e: host-to-host through the public API ---------------------------
    host = __import__("importlib").import_module("sparse-seam_b200.host")
    # Every rank expands its masks on the host, overlapping its copies; the
    # library's default for that is a quarter of the host's processors,
    # shared here among the ranks.
    unpack_threads = 0 if dist.world == 1 else \
        max(1, cpu_threads() // (4 * dist.world))
    hb = host.HostBatch(host_images, tile=tile, chunks=16,
                        persistent=False, packed=True,
                        threads=unpack_threads)
    # The host side needs more warm-up than the device: the first passes
    # after the buffers are set up run up to 40 % slower.  With one rank the
    # expansion's thread count is then picked by timing (it depends on the
    # host and on what else runs there).
    for _ in range(max(args.warmup, 10)):
        hb.run(stream)
    if dist.world == 1:
        hb.tune_threads(stream)
        for _ in range(2):
            hb.run(stream)
    stream.synchronize()
    hb.check()
    dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    end = None
    for _ in range(args.steps):
        end = hb.run(stream)
    end.synchronize()
    e2e_ms = dist.max(e0.elapsed_time(end))
    hb.check()
    import numpy as np
    bad = sum(int((hb.maxima[i] != maxs[i].cpu().numpy()).sum()) +
              int((hb.minima[i] != mins[i].cpu().numpy()).sum())
              for i in range(0, len(images), 25))
    out["e2e"] = {
        "value": round(dist.world * pixels * args.steps / (e2e_ms / 1e3)
                       / 1e9, 4),
        "unit": UNIT, "h2d_bytes_per_step": hb.h2d_bytes,
        "d2h_bytes_per_step": hb.d2h_bytes,
        "ms_per_step": round(e2e_ms / args.steps, 3),
        "api": ("sparse-seam_b200.host.HostBatch (ss_extrema_batch, 16 "
                "chunks; masks cross the bus as bit planes and are expanded "
                "into the pinned byte masks by host threads inside the "
                "timed region)"),
        "unpack_threads": hb.threads,
        "mismatches_vs_device_run": bad,
    }

    # -- CPU exact path on the host's cores (rank 0, N=1 only) -------------
    if dist.rank == 0 and dist.world == 1:
        threads = cpu_threads()
        cpix, ctimes = time_cpu_oracle(host_images, threads, reps=2)
        cval = cpix / min(ctimes) / 1e9
        out["cpu_baseline"] = {
            "value": round(cval, 5), "unit": UNIT, "cores": threads,
            "kind": "port",
            "sample": (f"the whole corpus ({cpix} px), union-find oracle "
                       "(oracle/ss_oracle.c), one image per thread, best "
                       "of 2"),
        }
        sample = [host_images[i] for i in (0, 1, 2, 3, 4)] + \
            [host_images[i] for i in range(len(images) - 5, len(images))]
        out["ref_protocol"] = ref_protocol_section(sample)
        out["reference_gpu"] = out["ref_protocol"]["t32"]["reference"]
    if large:
        out["launch_floor_2040x1356"] = launch_floor_section(
            pkg, images[0].device, stream, len(large), args.warmup,
            args.steps)
        out["single_image_passes_us"] = single_image_passes(
            pkg, images[large[0]], stream, args.warmup, 50, tile)
    return out


# ---------------------------------------------------------------------------
# Launch floor and the reference's per-image protocol
# ---------------------------------------------------------------------------

def _later_group(tiles: int, sms: int) -> int:
    """Tiles per CTA of the later passes, as the library chooses them."""
    group = 1
    while group < 32 and tiles > group * sms * 8:
        group *= 2
    return group


def launch_floor_section(pkg, device, stream, n_images, warmup, reps):
    """Graph replay of 1 and of 4 empty kernels per 2040x1356 image, with the
    grid shapes of the route's tile pass (the default row-scan CTAs, one tile
    per warp) and later passes (8 warps per CTA): the floor no launch-based
    per-image route goes below."""
    import torch
    lib = pkg.lib()
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    tiles = ((2040 + 31) // 32) * ((1356 + 31) // 32)
    cfg = pkg.get_kernel_config(32)
    warps = abs(cfg)
    per_cta = warps if cfg < 0 else 1     # row-scan: a tile per warp
    g1 = (tiles + per_cta - 1) // per_cta
    g2 = (tiles + _later_group(tiles, sms) - 1) // _later_group(tiles, sms)

    def run(k):
        s = ctypes.c_void_p(stream.cuda_stream)
        for _ in range(n_images):
            assert lib.ss_empty_launches(1, g1, 32 * warps, s) == 0
            if k > 1:
                assert lib.ss_empty_launches(k - 1, g2, 256, s) == 0

    out = {"grids": [g1, g2]}
    for k in (1, 4):
        ms = _graph_ms(lambda: run(k), stream, warmup, reps)
        out[f"us_{k}_launch"] = round(ms / n_images * 1e3, 3)
    return out


def single_image_passes(pkg, image, stream, warmup, reps, tile=32):
    """Device microseconds of each pass of the route on one image (graph of
    `reps` back-to-back launches of that pass; each pass is idempotent on a
    workspace where the earlier passes already ran)."""
    import torch
    mx = torch.empty_like(image)
    mn = torch.empty_like(image)
    plan = pkg.BatchPlan([image], [mx], [mn], tile=tile, stream=stream)
    ws = plan.make_workspace(stream=stream)
    plan.run(ws, stream=stream)
    stream.synchronize()
    out = {}
    for name, which in (("tile", 1), ("seam_flags", 4), ("resolve", 2)):
        def fn(w=which):
            for _ in range(reps):
                plan.run_pass(ws, w, stream=stream)
        out[name] = round(_graph_ms(fn, stream, 1, 1) / reps * 1e3, 3)
    ws.read_status(stream)
    return out


def _write_pgm(path, image):
    h, w = image.shape
    with open(path, "wb") as f:
        f.write(b"P5\n%d %d\n255\n" % (w, h))
        f.write(np.ascontiguousarray(image).tobytes())


def ref_protocol_section(sample, tiles=(32, 64), warmup=5, reps=30):
    """The product and the reference's own GPU routes on the same images with
    the reference's protocol (README.md:169-176 of the reference): per image
    `warmup` warm-ups and `reps` CUDA-event timed calls, no graph, median per
    image; aggregate = sum(px) / sum(median).  The product runs through the
    drop-in command-line harness (ss_harness, C ABI); the reference through
    its own harness routines built for sm_100a."""
    import csv
    import shutil
    import tempfile
    harness = os.path.join(ROOT, "sparse-seam_b200", "ss_harness")
    out = {"sample": f"{len(sample)} corpus images", "warmup": warmup,
           "reps": reps}
    tmp = tempfile.mkdtemp(prefix="ss_refproto_")
    try:
        src = os.path.join(tmp, "images")
        os.makedirs(src)
        for i, im in enumerate(sample):
            _write_pgm(os.path.join(src, f"img_{i:03d}.pgm"), im)
        for tile in tiles:
            dst = os.path.join(tmp, f"out_t{tile}")
            rc = subprocess.run(
                [harness, src, f"--output={dst}", f"--warmup={warmup}",
                 f"--reps={reps}", f"--tile={tile}"],
                capture_output=True, text=True, timeout=900).returncode
            entry = {}
            if rc != 0:
                entry["product"] = {"error": f"ss_harness exit {rc}"}
            else:
                with open(os.path.join(dst, "ss_harness.csv"),
                          newline="") as f:
                    rows = list(csv.DictReader(f))
                px = sum(int(r["width"]) * int(r["height"]) for r in rows)
                med = sum(float(r["median_compute_ms"]) for r in rows)
                h2h = sum(float(r["median_h2h_ms"]) for r in rows)
                entry["product"] = {"gpix_s": round(px / med / 1e6, 3),
                                    "h2h_gpix_s": round(px / h2h / 1e6, 3)}
            entry["reference"] = reference_gpu_routes(sample, tile, warmup,
                                                      reps)
            out[f"t{tile}"] = entry
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return out


# ---------------------------------------------------------------------------
# Batched uneven sizes, serving, resolution sweep
# ---------------------------------------------------------------------------

def _graph_ms(fn, stream, warmup: int, reps: int) -> float:
    """Device ms of one call of `fn`, captured in a CUDA graph and replayed
    back to back (CUDA events on `stream`)."""
    import torch
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(stream):
        fn()
        stream.synchronize()
        with torch.cuda.graph(g, stream=stream):
            fn()
    # Warm-up replays on the timing stream, and the device drained: a replay
    # left running on another stream would fall inside the timed window.
    with torch.cuda.stream(stream):
        for _ in range(max(1, warmup)):
            g.replay()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(reps):
            g.replay()
        e1.record(stream)
    e1.synchronize()
    del g
    return e0.elapsed_time(e1) / reps


def uneven_section(args, pkg, device, stream):
    """4096 images per batch, width and height drawn independently and
    log-uniformly from 64..1024, generators mixed 50 % smooth noise, 25 %
    uniform-quantised (2..256 levels), 25 % plateau maps.  Plain per-image
    launches against one batched launch (grid and persistent schedule) and the
    autotuned per-size-class batch, all graph-replayed; every image's masks
    are compared with its per-image result, and a sample with the oracle."""
    import torch
    from importlib import import_module
    import oracle
    synth = import_module("sparse-seam_b200.synth")
    at = import_module("sparse-seam_b200.autotune")
    images = synth.uneven_batch(4096, seed=20250, lo=64, hi=1024,
                                device=device)
    pixels = sum(im.numel() for im in images)
    ref_max = [torch.empty_like(i) for i in images]
    ref_min = [torch.empty_like(i) for i in images]
    maxs = [torch.empty_like(i) for i in images]
    mins = [torch.empty_like(i) for i in images]
    torch.cuda.synchronize()
    out = {"workload": ("4096 images, W and H log-uniform on 64..1024, "
                        "mixed generators (50 % smooth noise, 25 % "
                        "uniform-quantised, 25 % plateau maps), T=32"),
           "images": len(images), "pixels": pixels}

    big = max(images, key=lambda t: t.numel())
    ws1 = pkg.Workspace.for_image(big.shape[1], big.shape[0], 32)

    def per_image():
        for i, im in enumerate(images):
            pkg.extrema(im, 32, ref_max[i], ref_min[i], ws1, stream=stream)

    ms = _graph_ms(per_image, stream, args.warmup, args.steps)
    ws1.read_status(stream)
    out["per_image"] = {"gpix_s": round(pixels / ms / 1e6, 3),
                        "ms": round(ms, 4)}

    plan = pkg.BatchPlan(images, maxs, mins, tile=32, stream=stream)
    ws = plan.make_workspace(stream=stream)
    for persistent in (False, True):
        ms = _graph_ms(lambda: plan.run(ws, persistent=persistent,
                                        stream=stream),
                       stream, args.warmup, args.steps)
        ws.read_status(stream)
        key = "batched_persistent" if persistent else "batched_grid"
        out[key] = {"gpix_s": round(pixels / ms / 1e6, 3), "ms": round(ms, 4)}
    bad = sum(int((a != b).sum()) for a, b in
              zip(maxs + mins, ref_max + ref_min))

    import time as _time
    t0 = _time.time()
    table = at.tune(pixels_per_class=8 << 20, reps=3, seed=7, device=device)
    tune_s = _time.time() - t0
    for m in maxs + mins:
        m.fill_(3)
    tb = at.TunedBatch(images, maxs, mins, table, stream=stream)
    ms = _graph_ms(lambda: tb.run(stream=stream), stream, args.warmup,
                   args.steps)
    tb.read_status(stream)
    bad += sum(int((a != b).sum()) for a, b in
               zip(maxs + mins, ref_max + ref_min))
    out["autotuned"] = {
        "gpix_s": round(pixels / ms / 1e6, 3), "ms": round(ms, 4),
        "launches": 1 if tb.single is not None else len(tb.parts),
        "form": tb.form,
        "forms_ms": tb.timings_ms,
        "tuning_s": round(tune_s, 1),
        "choices": {str(k): v.label() for k, v in table.choices.items()},
        "mix_choice": table.mix.label() if table.mix else None,
        "class_bounds_px": list(at.CLASS_BOUNDS[:-1]),
    }
    sample = list(range(0, len(images), 64))
    want = oracle.extrema_batch([images[i].cpu().numpy() for i in sample],
                                threads=cpu_threads())
    for j, i in enumerate(sample):
        bad += int((maxs[i].cpu().numpy() != want[0][j]).sum())
        bad += int((mins[i].cpu().numpy() != want[1][j]).sum())
    out["mismatches"] = bad
    out["checked"] = (f"all {len(images)} images against their per-image "
                      f"masks, {len(sample)} against the oracle")
    return out


SERVE_SIZES = ((321, 481), (1024, 1024), (1356, 2040), (4096, 4096),
               (8192, 8192))
SERVE_WEIGHTS = (0.3, 0.3, 0.2, 0.15, 0.05)
SERVE_RATES = (50.0, 100.0, 500.0, 2000.0)   # requests per second
SERVE_COUNTS = (8, 8, 8, 4, 4)   # distinct images per request size


def serve_plateau_jobs():
    """(size index, image index, seed) of the served stream's plateau maps."""
    return [(k, j, 1000 * k + j) for k in range(len(SERVE_SIZES))
            for j in range(SERVE_COUNTS[k]) if j % 4 == 3]


def start_plateau_maps():
    """Starts the served stream's plateau maps (distance maps of 8192^2
    ellipse masks take tens of seconds on the host) in spawned worker
    processes, so they are ready when the serving section starts."""
    import concurrent.futures
    import multiprocessing
    from importlib import import_module
    synth = import_module("sparse-seam_b200.synth")
    ex = concurrent.futures.ProcessPoolExecutor(
        max_workers=4, mp_context=multiprocessing.get_context("spawn"))
    futures = {(k, j): ex.submit(synth.plateau_map, *SERVE_SIZES[k], seed)
               for k, j, seed in serve_plateau_jobs()}
    return ex, futures


def _serve_images(device, plateau):
    """Distinct pinned host images per request size, the generators of the
    single-image, corpus and uneven-batch workloads in turn: uniform 16
    levels, smooth noise, uniform-quantised (2..256 levels), plateau maps."""
    import torch
    from importlib import import_module
    synth = import_module("sparse-seam_b200.synth")
    pool = {}
    for k, (h, w) in enumerate(SERVE_SIZES):
        imgs = []
        for j in range(SERVE_COUNTS[k]):
            kind = j % 4
            seed = 1000 * k + j
            if kind == 0:
                t = torch.from_numpy(synth.uniform_q16(h, w, seed))
            elif kind == 1:
                t = synth.smooth_noise(h, w, seed, device=device).cpu()
            elif kind == 2:
                rng = np.random.default_rng(seed)
                levels = int(rng.integers(2, 257))
                t = torch.from_numpy(synth.quantize(
                    rng.integers(0, 256, size=(h, w)).astype(np.uint8),
                    levels))
            else:
                t = torch.from_numpy(plateau[(k, j)].result())
            p = torch.empty((h, w), dtype=torch.uint8, pin_memory=True)
            p.copy_(t)
            imgs.append(p)
        pool[k] = imgs
    return pool


def serving_section(args, pkg, device, stream, plateau):
    """Served request stream: Poisson arrivals, each request one host image
    whose size is drawn from 481x321 / 1024^2 / 2040x1356 / 4096^2 / 8192^2
    (weights 0.3 / 0.3 / 0.2 / 0.15 / 0.05).  Latency = completion (masks in
    the caller's pinned host buffers) minus scheduled arrival.  Also the
    saturated throughput (every request at t = 0) against plain per-image
    host-to-host calls (copy in, ss_extrema, copy out, wait) on the same
    requests, and a mixed burst whose every result is compared with the same
    image's result alone."""
    import torch
    from importlib import import_module
    serve = import_module("sparse-seam_b200.serve")
    pool = _serve_images(device, plateau)
    ring = {0: 16, 1: 16, 2: 12, 3: 8, 4: 4}
    outs = {k: [(torch.empty(SERVE_SIZES[k], dtype=torch.uint8,
                             pin_memory=True),
                 torch.empty(SERVE_SIZES[k], dtype=torch.uint8,
                             pin_memory=True)) for _ in range(ring[k])]
            for k in range(len(SERVE_SIZES))}
    rng = np.random.default_rng(55)

    def draw(n):
        ks = rng.choice(len(SERVE_SIZES), size=n, p=SERVE_WEIGHTS)
        return [(int(k), int(rng.integers(0, len(pool[int(k)]))))
                for k in ks]

    def maker(reqs):
        used = {k: 0 for k in range(len(SERVE_SIZES))}

        def make(i):
            k, j = reqs[i]
            o = outs[k][used[k] % ring[k]]
            used[k] += 1
            return pool[k][j], o[0], o[1]
        return make

    cfg = dict(tile=32, persistent=True, inflight=3, max_batch_images=256,
               batch_tiles=1 << 17, pool_bytes=8 << 30)
    out = {"workload": ("Poisson arrivals at 50 / 100 / 500 / 2000 req/s; "
                        "request sizes 481x321 / 1024^2 / 2040x1356 / "
                        "4096^2 / 8192^2 with weights 0.3/0.3/0.2/0.15/0.05; "
                        "generators in turn uniform 16 levels, smooth noise, "
                        "uniform-quantised 2..256 levels, plateau maps; "
                        "pinned host images in, masks out to pinned host "
                        "buffers"),
           "duration_s": float(args.serve_seconds),
           "server": {k: v for k, v in cfg.items()}}
    rates = {}
    with serve.Server(**cfg) as srv:
        warm = draw(24)
        serve.run_trace(srv, np.zeros(len(warm), dtype=np.int64),
                        maker(warm))
        dur = float(args.serve_seconds)
        for rate in SERVE_RATES:
            arrivals = serve.poisson_trace(rate, dur, seed=int(rate))
            reqs = draw(len(arrivals))
            res = serve.run_trace(srv, arrivals, maker(reqs))
            d = res.as_dict()
            d.pop("stats")
            d["offered_gpix_s"] = round(
                rate * float(np.dot(SERVE_WEIGHTS,
                                    [h * w for h, w in SERVE_SIZES])) / 1e9,
                3)
            rates[str(int(rate))] = d
        # Saturated: every request arrives at once.
        sat = draw(300)
        res = serve.run_trace(srv, np.zeros(len(sat), dtype=np.int64),
                              maker(sat))
        out["saturated"] = {k: v for k, v in res.as_dict().items()
                            if k != "stats"}
        out["server_stats"] = srv.stats()
    out["rates_req_s"] = rates

    # Plain per-image host-to-host calls on the same saturated request list.
    big_ws = pkg.Workspace.for_image(8192, 8192, 32)
    dev_in = torch.empty((8192, 8192), dtype=torch.uint8, device=device)
    dev_mx = torch.empty_like(dev_in)
    dev_mn = torch.empty_like(dev_in)
    px = 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for k, j in sat:
            h, w = SERVE_SIZES[k]
            im = pool[k][j]
            d_in = dev_in.view(-1)[:h * w].view(h, w)
            d_mx = dev_mx.view(-1)[:h * w].view(h, w)
            d_mn = dev_mn.view(-1)[:h * w].view(h, w)
            d_in.copy_(im, non_blocking=True)
            pkg.extrema(d_in, 32, d_mx, d_mn, big_ws, stream=stream)
            o = outs[k][0]
            o[0].copy_(d_mx, non_blocking=True)
            o[1].copy_(d_mn, non_blocking=True)
            stream.synchronize()
            px += h * w
        e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    big_ws.read_status(stream)
    out["per_image_h2h"] = {"gpix_s": round(px / ms / 1e6, 3),
                            "ms": round(ms, 2), "requests": len(sat)}

    # Mixed burst, distinct outputs: each result against the image alone.
    burst = [(k, j) for k in range(len(SERVE_SIZES))
             for j in range(min(2, len(pool[k])))] + draw(12)
    bouts = [(torch.empty(SERVE_SIZES[k], dtype=torch.uint8, pin_memory=True),
              torch.empty(SERVE_SIZES[k], dtype=torch.uint8, pin_memory=True))
             for k, _ in burst]
    with serve.Server(**cfg) as srv:
        for i, (k, j) in enumerate(burst):
            srv.submit(pool[k][j], *bouts[i], user=i)
        done = []
        while len(done) < len(burst):
            done.extend(srv.poll(timeout_us=100_000))
    bad = sum(1 for c in done if c.status != 0)
    for i, (k, j) in enumerate(burst):
        h, w = SERVE_SIZES[k]
        d_in = pool[k][j].to(device)
        mx, mn = pkg.extrema(d_in, 32)
        bad += int((mx.cpu() != bouts[i][0]).sum())
        bad += int((mn.cpu() != bouts[i][1]).sum())
    out["mix_vs_alone_mismatches"] = bad
    out["mix_requests"] = len(burst)
    return out


def resolution_section(args, pkg, device, stream, hbm):
    """Single smooth-noise images from 1 Mpixel to 16384^2 (268 Mpixel):
    device-resident ss_extrema, graph-replayed; each checked against the
    oracle's row-band route."""
    import torch
    from importlib import import_module
    import oracle
    synth = import_module("sparse-seam_b200.synth")
    out = {}
    for side in (1024, 2048, 4096, 8192, 16384):
        img = synth.smooth_noise(side, side, seed=side, device=device)
        mx = torch.empty_like(img)
        mn = torch.empty_like(img)
        ws = pkg.Workspace.for_image(side, side, 32)
        reps = max(3, min(args.steps, 20))
        ms = _graph_ms(lambda: pkg.extrema(img, 32, mx, mn, ws,
                                           stream=stream),
                       stream, args.warmup, reps)
        ws.read_status(stream)
        want = oracle.extrema(img.cpu().numpy(), method="bands",
                              threads=cpu_threads())
        bad = int((mx.cpu().numpy() != want[0]).sum()) + \
            int((mn.cpu().numpy() != want[1]).sum())
        px = side * side
        out[f"{side}x{side}"] = {
            "us": round(ms * 1e3, 2), "gpix_s": round(px / ms / 1e6, 3),
            "roofline_frac": round(BYTES_PER_PIXEL * px / (ms / 1e3) / 1e9
                                   / hbm, 4),
            "mismatches": bad}
        del img, mx, mn, ws, want
        torch.cuda.empty_cache()
    return out


if __name__ == "__main__":
    sys.exit(main())
