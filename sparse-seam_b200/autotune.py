"""Batch autotuner: per image-size class, the tile, kernel family, schedule,
seam/resolve grouping and fragment flatten schedule that run a batch fastest
on this GPU.

The reference fixes its tile size and classify threads at compile time and
sweeps them with a separate benchmark binary
(harness/configuration_study/sparse_config_benchmark_v0_8.cu:17-30).  Here the
choice is made at run time, per size class, by timing candidate launches
(``ss_extrema_batch_launch``) on a seeded synthetic batch of that class with
CUDA events.  No choice changes the masks: every candidate's masks are checked
byte-equal to the first candidate's before its time is accepted.

A class is a range of image areas (pixels).  Besides the classes, the
candidates are timed on a "mix": a seeded batch drawn like an uneven-size
batch (sides log-uniform on 64..1024, mixed generators), whose best choice
is the one for a whole batch in one launch.  `TunedBatch` times, on its own
batch, the split by class, one launch with the mix's choice and one default
launch, and runs the fastest.
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
    flatten: int = 0  # row-scan fragment flatten schedule (ss_launch.flatten)

    def label(self) -> str:
        kind = f"rowscan{-self.warps}" if self.warps < 0 else \
            f"cta{self.warps}"
        return (f"T{self.tile}-{kind}-{'persistent' if self.persistent else 'grid'}"
                f"-g{self.group}-f{self.flatten}")

    def is_default(self) -> bool:
        return (self.tile == 32 and
                self.warps == _pkg.get_kernel_config(32) and
                not self.persistent and self.group == 0 and self.flatten == 0)


# Row-scan seam/resolve groupings and flatten schedules tried.
GROUPS = (0, 4, 32)
FLATTENS = (0, 1, 2)


def candidates() -> List[Choice]:
    """Every launch choice the library offers (the CTA-per-tile kernels with
    the grid schedule only: they are an order of magnitude slower)."""
    out = []
    for tile, family in _pkg.KERNEL_CONFIGS.items():
        for warps in family:
            if warps > 0:
                out.append(Choice(tile, warps, False, 0))
                continue
            for persistent in (False, True):
                for group in GROUPS:
                    for flatten in FLATTENS:
                        out.append(Choice(tile, warps, persistent, group,
                                          flatten))
    # The library's defaults first: they are the comparison baseline.
    default = [c for c in out if c.is_default()]
    return default + [c for c in out if c not in default]


@dataclass
class TuningTable:
    choices: Dict[int, Choice]
    timings_ms: Dict[int, Dict[str, float]]
    mix: Optional[Choice] = None             # best on the mixed batch
    mix_timings_ms: Optional[Dict[str, float]] = None

    def choice_for(self, height: int, width: int) -> Choice:
        return self.choices[size_class(height, width)]

    def to_json(self) -> str:
        return json.dumps({
            "class_bounds": list(CLASS_BOUNDS),
            "choices": {str(k): asdict(v) for k, v in self.choices.items()},
            "timings_ms": {str(k): v for k, v in self.timings_ms.items()},
            "mix": asdict(self.mix) if self.mix else None,
            "mix_timings_ms": self.mix_timings_ms,
        })

    @staticmethod
    def from_json(text: str) -> "TuningTable":
        data = json.loads(text)
        if list(data["class_bounds"]) != list(CLASS_BOUNDS):
            raise ValueError("table was tuned for other size classes")
        mix = data.get("mix")
        return TuningTable(
            {int(k): Choice(**v) for k, v in data["choices"].items()},
            {int(k): v for k, v in data.get("timings_ms", {}).items()},
            Choice(**mix) if mix else None, data.get("mix_timings_ms"))


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
                                  group=choice.group,
                                  flatten=choice.flatten, stream=stream)
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


def mix_sample(count: int, seed: int, device) -> List:
    """Seeded images drawn like an uneven-size batch: width and height
    log-uniform on 64..1024, mixed generators."""
    synth = importlib.import_module(__package__ + ".synth")
    return synth.uneven_batch(count, seed=seed, lo=64, hi=1024, device=device)


def _time_all(images, cands, reps, stream, what):
    """Milliseconds of every candidate on `images`; raises if a candidate's
    masks differ from the first's."""
    import torch
    ref = None
    out: Dict[Choice, float] = {}
    for c in cands:
        ms, mx, mn = _time_choice(images, c, reps, stream)
        if ref is None:
            ref = (mx, mn)
        else:
            for a, b in zip(ref[0] + ref[1], mx + mn):
                if not torch.equal(a, b):
                    raise RuntimeError(f"{what}: {c.label()} changed the masks")
        out[c] = ms
    return out


def tune(pixels_per_class: int = 16 << 20, reps: int = 5, seed: int = 0,
         device="cuda", classes: Optional[Sequence[int]] = None,
         choices: Optional[Sequence[Choice]] = None,
         mix_images: int = 384) -> TuningTable:
    """Times every candidate on a synthetic batch of each class; picks the
    candidate fastest over all classes, and for a class its own fastest if
    that beats the common one by MARGIN.  Also times every candidate on a
    mixed uneven-size batch of `mix_images` images (0: skipped) and keeps the
    fastest as the table's `mix` choice.  Raises if any candidate's masks
    differ from the first's."""
    import torch
    stream = torch.cuda.Stream()
    cands = list(choices) if choices else candidates()
    picked: Dict[int, Choice] = {}
    timings: Dict[int, Dict[str, float]] = {}
    raw: Dict[int, Dict[Choice, float]] = {}
    for k in (classes if classes is not None else range(len(CLASS_BOUNDS))):
        images = class_sample(k, pixels_per_class, seed + 7919 * k, device)
        raw[k] = _time_all(images, cands, reps, stream, f"class {k}")
        timings[k] = {c.label(): round(ms, 4) for c, ms in raw[k].items()}
    mix = None
    mix_timings = None
    if mix_images:
        images = mix_sample(mix_images, seed + 104729, device)
        t = _time_all(images, cands, reps, stream, "mix")
        mix = min(cands, key=lambda c: (t[c], cands.index(c)))
        mix_timings = {c.label(): round(ms, 4) for c, ms in t.items()}
    # One choice for every class unless a class gains more than MARGIN from
    # its own best: every distinct choice is one more launch of the batch.
    common = min(cands, key=lambda c: (sum(t[c] for t in raw.values()),
                                       cands.index(c)))
    for k, t in raw.items():
        own = min(t, key=t.get)
        picked[k] = own if t[own] < t[common] * (1.0 - MARGIN) else common
    return TuningTable(picked, timings, mix, mix_timings)


class TunedBatch:
    """A batch run in the fastest of three forms, chosen by timing each on
    this batch once, at construction:

      split    the batch split by size class, each part launched with its
               class's tuned choice (parts on their own streams, forked from
               and joined back into the caller's stream with events, so the
               GPU fills its SMs from all parts at once; classes whose
               choices differ only in the seam/resolve grouping share one
               launch);
      mix      one launch over the whole batch with the table's `mix` choice
               (tuned on a mixed uneven-size batch);
      default  one launch over the whole batch with the library defaults.

    `form` names the one `run` uses.  The fork and join are captured into a
    CUDA graph like any other stream work.
    """

    def __init__(self, images: Sequence, maxima: Sequence, minima: Sequence,
                 table: TuningTable, stream=None):
        import torch
        parts: Dict[Choice, List[int]] = {}
        groups: Dict[Tuple[int, int, bool, int], set] = {}
        for c in table.choices.values():
            groups.setdefault((c.tile, c.warps, c.persistent, c.flatten),
                              set()).add(c.group)
        for i, im in enumerate(images):
            c = table.choice_for(*im.shape)
            key = (c.tile, c.warps, c.persistent, c.flatten)
            if len(groups[key]) > 1:
                c = Choice(c.tile, c.warps, c.persistent, 0, c.flatten)
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
        # Whole-batch launches: the mix's choice and the default.
        self.single: Optional[Tuple[Choice, object, object]] = None
        self.form = "split"
        self.timings_ms: Dict[str, float] = {}
        if not self.parts:
            return
        main = stream or torch.cuda.current_stream()
        forms = {}
        if len(self.parts) > 1 or not self.parts[0][0].is_default():
            forms["split"] = (None, self._run_parts)
        default = Choice(32, _pkg.get_kernel_config(32), False, 0, 0)
        wholes = [("default", default)]
        if table.mix is not None and table.mix != default:
            wholes.append(("mix", table.mix))
        built = {}
        for name, choice in wholes:
            plan = _pkg.BatchPlan(list(images), list(maxima), list(minima),
                                  tile=choice.tile, stream=stream)
            ws = plan.make_workspace(stream=stream)
            built[name] = (choice, plan, ws)
            forms[name] = (built[name], None)
        for name, (whole, fn) in forms.items():
            if whole is not None:
                choice, plan, ws = whole
                fn = (lambda s, c=choice, p=plan, w=ws:  # noqa: E731
                      p.run_launch(w, warps=c.warps, persistent=c.persistent,
                                   group=c.group, flatten=c.flatten, stream=s))
            self.timings_ms[name] = round(_time_on(main, fn), 4)
        self.form = min(self.timings_ms, key=self.timings_ms.get)
        if self.form != "split":
            self.single = built[self.form]

    def run(self, stream=None) -> None:
        import torch
        main = stream or torch.cuda.current_stream()
        if self.single is not None:
            c, plan, ws = self.single
            plan.run_launch(ws, warps=c.warps, persistent=c.persistent,
                            group=c.group, flatten=c.flatten, stream=main)
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
                            flatten=choice.flatten, stream=st)
            if i:
                done = torch.cuda.Event()
                done.record(st)
                joins.append(done)
        for done in joins:
            main.wait_event(done)

    def read_status(self, stream=None) -> None:
        if self.single is not None:
            self.single[2].read_status(stream)
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
