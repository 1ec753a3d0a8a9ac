"""Batch autotuner: per image-size class, the tile, kernel family, schedule and
seam/resolve grouping that run a batch fastest on this GPU.

The reference fixes its tile size and classify threads at compile time and
sweeps them with a separate benchmark binary
(harness/configuration_study/sparse_config_benchmark_v0_8.cu:17-30).  Here the
choice is made at run time, per size class, by timing candidate launches
(``ss_extrema_batch_launch``) on a seeded synthetic batch of that class with
CUDA events.  No choice changes the masks: every candidate's masks are checked
byte-equal to the first candidate's before its time is accepted.

A class is a range of image areas (pixels).  `TunedBatch` splits a batch by
class and runs one launch per class with that class's choice.
"""
from __future__ import annotations

import importlib
import json
from dataclasses import asdict, dataclass
from typing import Dict, List, Optional, Sequence, Tuple

_pkg = importlib.import_module(__package__)

# Upper bounds (exclusive) of the area classes, in pixels.
CLASS_BOUNDS = (64 * 64 * 4, 256 * 256, 512 * 512, 1 << 40)


def size_class(height: int, width: int) -> int:
    area = int(height) * int(width)
    for k, bound in enumerate(CLASS_BOUNDS):
        if area < bound:
            return k
    return len(CLASS_BOUNDS) - 1


@dataclass(frozen=True)
class Choice:
    tile: int
    warps: int        # ss_set_kernel_config value (negative: row-scan)
    persistent: bool
    group: int        # row-scan seam/resolve tiles per warp, 0 = automatic

    def label(self) -> str:
        kind = f"rowscan{-self.warps}" if self.warps < 0 else \
            f"cta{self.warps}"
        return (f"T{self.tile}-{kind}-{'persistent' if self.persistent else 'grid'}"
                f"-g{self.group}")


def candidates() -> List[Choice]:
    """Every launch choice the library offers."""
    out = []
    for tile, family in _pkg.KERNEL_CONFIGS.items():
        for warps in family:
            for persistent in (False, True):
                groups = (0, 1, 4, 32) if warps < 0 else (0,)
                for group in groups:
                    out.append(Choice(tile, warps, persistent, group))
    # The library's defaults first: they are the comparison baseline.
    default = [c for c in out if c.tile == 32 and
               c.warps == _pkg.get_kernel_config(32) and not c.persistent and
               c.group == 0]
    return default + [c for c in out if c not in default]


@dataclass
class TuningTable:
    choices: Dict[int, Choice]
    timings_ms: Dict[int, Dict[str, float]]

    def choice_for(self, height: int, width: int) -> Choice:
        return self.choices[size_class(height, width)]

    def to_json(self) -> str:
        return json.dumps({
            "class_bounds": list(CLASS_BOUNDS),
            "choices": {str(k): asdict(v) for k, v in self.choices.items()},
            "timings_ms": {str(k): v for k, v in self.timings_ms.items()},
        })

    @staticmethod
    def from_json(text: str) -> "TuningTable":
        data = json.loads(text)
        if list(data["class_bounds"]) != list(CLASS_BOUNDS):
            raise ValueError("table was tuned for other size classes")
        return TuningTable(
            {int(k): Choice(**v) for k, v in data["choices"].items()},
            {int(k): v for k, v in data.get("timings_ms", {}).items()})


def class_sample(k: int, pixels: int, seed: int, device) -> List:
    """Seeded mixed-generator images whose areas fall in class k."""
    synth = importlib.import_module(__package__ + ".synth")
    lo = 0 if k == 0 else CLASS_BOUNDS[k - 1]
    hi = CLASS_BOUNDS[k] if k + 1 < len(CLASS_BOUNDS) else 2048 * 2048
    # Side ranges that make most drawn sizes fall in the class.
    side_lo, side_hi = ((32, 160), (96, 320), (224, 640), (512, 2048))[k]
    imgs, total, s = [], 0, seed
    while total < pixels:
        batch = synth.uneven_batch(64, seed=s, lo=side_lo, hi=side_hi,
                                   device=device)
        s += 1
        for im in batch:
            a = im.shape[0] * im.shape[1]
            if max(lo, 1) <= a < hi:
                imgs.append(im)
                total += a
                if total >= pixels:
                    break
    return imgs


def _time_choice(images, choice: Choice, reps: int, stream):
    import torch
    maxs = [torch.empty_like(i) for i in images]
    mins = [torch.empty_like(i) for i in images]
    plan = _pkg.BatchPlan(images, maxs, mins, tile=choice.tile, stream=stream)
    ws = plan.make_workspace(stream=stream)
    run = lambda: plan.run_launch(ws, warps=choice.warps,       # noqa: E731
                                  persistent=choice.persistent,
                                  group=choice.group, stream=stream)
    with torch.cuda.stream(stream):
        run()
        run()
    ws.read_status(stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        run()
    e1.record(stream)
    e1.synchronize()
    ws.read_status(stream)
    return e0.elapsed_time(e1) / reps, maxs, mins


# A class keeps its own best choice only when it beats the choice that is
# best over all classes by at least this much: smaller gaps are within
# run-to-run noise, and one common choice keeps the batch in one launch.
MARGIN = 0.03


def tune(pixels_per_class: int = 16 << 20, reps: int = 5, seed: int = 0,
         device="cuda", classes: Optional[Sequence[int]] = None,
         choices: Optional[Sequence[Choice]] = None) -> TuningTable:
    """Times every candidate on a synthetic batch of each class; picks the
    candidate fastest over all classes, and for a class its own fastest if
    that beats the common one by MARGIN.  Raises if any candidate's masks
    differ from the first's."""
    import torch
    stream = torch.cuda.Stream()
    cands = list(choices) if choices else candidates()
    picked: Dict[int, Choice] = {}
    timings: Dict[int, Dict[str, float]] = {}
    raw: Dict[int, Dict[Choice, float]] = {}
    for k in (classes if classes is not None else range(len(CLASS_BOUNDS))):
        images = class_sample(k, pixels_per_class, seed + 7919 * k, device)
        ref = None
        timings[k] = {}
        raw[k] = {}
        for c in cands:
            ms, mx, mn = _time_choice(images, c, reps, stream)
            if ref is None:
                ref = (mx, mn)
            else:
                for a, b in zip(ref[0] + ref[1], mx + mn):
                    if not torch.equal(a, b):
                        raise RuntimeError(
                            f"class {k}: {c.label()} changed the masks")
            timings[k][c.label()] = round(ms, 4)
            raw[k][c] = ms
    # One choice for every class unless a class gains more than MARGIN from
    # its own best: every distinct choice is one more launch of the batch.
    common = min(cands, key=lambda c: (sum(t[c] for t in raw.values()),
                                       cands.index(c)))
    for k, t in raw.items():
        own = min(t, key=t.get)
        picked[k] = own if t[own] < t[common] * (1.0 - MARGIN) else common
    return TuningTable(picked, timings)


class TunedBatch:
    """A batch split by size class, each part launched with its tuned choice.

    Classes whose choices differ only in the seam/resolve grouping share one
    launch (with the grouping chosen from that launch's tile count).  The
    parts run concurrently, each on its own stream forked from and joined
    back into the caller's stream with events, so the GPU fills its SMs from
    all parts at once; the fork and join are captured into a CUDA graph like
    any other stream work.  When the batch splits into several parts, the
    split and one launch over the whole batch are timed on it once, at
    construction, and `run` uses the faster form (`single` is set when that
    is the one launch).  The same check guards a one-part batch whose tuned
    choice is not the library default.
    """

    def __init__(self, images: Sequence, maxima: Sequence, minima: Sequence,
                 table: TuningTable, stream=None):
        import torch
        parts: Dict[Choice, List[int]] = {}
        groups: Dict[Tuple[int, int, bool], set] = {}
        for c in table.choices.values():
            groups.setdefault((c.tile, c.warps, c.persistent), set()).add(
                c.group)
        for i, im in enumerate(images):
            c = table.choice_for(*im.shape)
            key = (c.tile, c.warps, c.persistent)
            if len(groups[key]) > 1:
                c = Choice(c.tile, c.warps, c.persistent, 0)
            parts.setdefault(c, []).append(i)
        self.parts: List[Tuple[Choice, object, object]] = []
        for choice, idx in sorted(parts.items(), key=lambda kv: kv[0].label()):
            plan = _pkg.BatchPlan([images[i] for i in idx],
                                  [maxima[i] for i in idx],
                                  [minima[i] for i in idx], tile=choice.tile,
                                  stream=stream)
            self.parts.append((choice, plan,
                               plan.make_workspace(stream=stream)))
        device = images[0].device if len(images) else None
        self._streams = [torch.cuda.Stream(device)
                         for _ in self.parts[1:]]
        # Choices tuned on one class's sample at a time need not carry over
        # to this batch (a seam/resolve grouping fitted to the sample's
        # launch size, or a split slower than one launch): unless the tuned
        # form is already the library default over the whole batch, both are
        # timed on the batch once and the faster is kept.
        self.single = None
        default = (len(self.parts) == 1 and
                   self.parts[0][0].warps == _pkg.get_kernel_config(
                       self.parts[0][0].tile) and
                   not self.parts[0][0].persistent and
                   self.parts[0][0].group == 0)
        if self.parts and not default:
            tiles = [c.tile for c in table.choices.values()]
            tile = max(set(tiles), key=tiles.count) if tiles else 32
            plan = _pkg.BatchPlan(list(images), list(maxima), list(minima),
                                  tile=tile, stream=stream)
            ws = plan.make_workspace(stream=stream)
            main = stream or torch.cuda.current_stream()
            t_split = _time_on(main, self._run_parts)
            t_single = _time_on(main, lambda s: plan.run(ws, stream=s))
            if t_single < t_split:
                self.single = (plan, ws)

    def run(self, stream=None) -> None:
        import torch
        main = stream or torch.cuda.current_stream()
        if self.single is not None:
            plan, ws = self.single
            plan.run(ws, stream=main)
            return
        self._run_parts(main)

    def _run_parts(self, main) -> None:
        import torch
        fork = torch.cuda.Event()
        fork.record(main)
        joins = []
        for i, (choice, plan, ws) in enumerate(self.parts):
            st = main if i == 0 else self._streams[i - 1]
            if i:
                st.wait_event(fork)
            plan.run_launch(ws, warps=choice.warps,
                            persistent=choice.persistent, group=choice.group,
                            stream=st)
            if i:
                done = torch.cuda.Event()
                done.record(st)
                joins.append(done)
        for done in joins:
            main.wait_event(done)

    def read_status(self, stream=None) -> None:
        if self.single is not None:
            self.single[1].read_status(stream)
            return
        for _, _, ws in self.parts:
            ws.read_status(stream)


def _time_on(stream, fn, reps: int = 3) -> float:
    """Device milliseconds of one call of fn(stream), after one warm-up."""
    import torch
    fn(stream)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(reps):
        fn(stream)
    end.record(stream)
    end.synchronize()
    return start.elapsed_time(end) / reps
