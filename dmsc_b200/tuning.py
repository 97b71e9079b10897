"""Autotuner of the launch shapes (no counterpart in the reference, whose CPU
path fixes its blocking at compile time: cpu/gradient.hxx:15
DEFAULT_GRADIENT_BLOCK_SIZE, cpu/cell_groups.hxx:9 CACHE_DEPTH).

Tunables (``dmsc_b200_set_tuning`` in include/dmsc_b200.h), none of which
changes an output bit:

* ``grad_shape``: gradient tile of 32 index columns x 31, 63 or 127 rows
  (how much of the value window and its halo row each CTA stages), or the
  persistent kernel whose tile windows are staged by tensor-memory copies
  (63 or 127 rows);
* ``label_shape``: 64 x 64 label tiles on 1024 or 512 threads (4 or 8 cells
  per thread in the barrier-free pointer jumping);
* ``pair_shape``: pairing items each thread advances together (2 or 4,
  with 5 or 4 resident blocks per SM);
* ``replay_shape``: replay cancellations each thread advances together (1 or
  2, with 4 or 3 resident blocks per SM);
* ``emit_shape``: geometry-expansion chain tasks each thread advances
  together (1 or 2, with 5 or 3 resident blocks per SM);
* ``pair_blocks_per_sm``, ``replay_blocks_per_sm``, ``emit_blocks_per_sm``:
  resident blocks per SM of the three persistent round loops (0 = all that
  fit); fewer blocks make each grid barrier cheaper, more hide more latency;
* ``seg_cursors``: raw-arc walks per lane of the segment writer (1 or 2).

``tune`` sweeps one tunable at a time on the caller's own input (coordinate
descent in the order above), timing the stage that tunable affects with the
library's CUDA events, ``reps`` runs per candidate, and keeps the candidate
with the smallest median. The choice is cached per device and image-size
class (total pixels of a call, rounded down to a power of two) and applied to
every later call of that class on that device; a class never tuned runs the
default shapes.
"""

from __future__ import annotations

import math
import statistics
import threading

import torch

from . import _lib

# tunable, the stage it affects, candidates from the device limits
TUNABLES = (
    ("grad_shape", "gradient", lambda lim: list(range(lim["grad_shapes"]))),
    ("label_shape", "labels", lambda lim: list(range(lim["label_shapes"]))),
    ("pair_shape", "pairing", lambda lim: list(range(lim["pair_shapes"]))),
    ("pair_blocks_per_sm", "pairing", lambda lim: _blocks(lim["pair_blocks_per_sm"])),
    ("replay_shape", "replay", lambda lim: list(range(lim["replay_shapes"]))),
    ("replay_blocks_per_sm", "replay", lambda lim: _blocks(lim["replay_blocks_per_sm"])),
    ("emit_shape", "fetch_geometry", lambda lim: list(range(lim["emit_shapes"]))),
    ("emit_blocks_per_sm", "fetch_geometry", lambda lim: _blocks(lim["emit_blocks_per_sm"])),
    ("seg_cursors", "fetch_geometry", lambda lim: list(range(1, lim["seg_cursors"] + 1))),
)

_lock = threading.Lock()
_cache: dict = {}  # (device, size class) -> {tunable: value}
_tuning = threading.local()  # set while tune() runs on this thread


def _default_tuning() -> dict:
    return {"grad_shape": 3, "label_shape": 1, "pair_shape": 0, "pair_blocks_per_sm": 0, "replay_shape": 0,
            "replay_blocks_per_sm": 0, "emit_shape": 0,
            "emit_blocks_per_sm": 0, "seg_cursors": 1}


def _blocks(most: int) -> list:
    """Candidates for a persistent kernel: all that fit (0), then 1, 2, 4 ...
    blocks per SM below that."""
    out, b = [0], 1
    while b < most:
        out.append(b)
        b *= 2
    return out


def size_class(npx: int) -> int:
    """Image-size class of a call: floor(log2(total pixels))."""
    return int(math.floor(math.log2(max(1, int(npx)))))


def select(timings: dict):
    """Candidate with the smallest median time; ties keep the earliest
    candidate (the default comes first). ``timings``: candidate -> list of
    times (ms)."""
    best, best_t = None, None
    for cand, ts in timings.items():
        if not ts:
            continue
        m = statistics.median(ts)
        if best_t is None or m < best_t:
            best, best_t = cand, m
    return best


def choice(device: int, npx: int):
    """Cached choice of a device and size class, or None."""
    with _lock:
        return dict(_cache.get((device, size_class(npx)), {})) or None


def apply(ctx, npx: int) -> None:
    """Sets the launch shapes of this call's size class on the context: the
    cached choice, or the defaults when the class was never tuned. A no-op
    while tune() sweeps on this thread."""
    if getattr(_tuning, "active", False):
        return
    c = choice(ctx.device, npx)
    want = c if c is not None else _default_tuning()
    if getattr(ctx, "_applied_tuning", None) != want:
        ctx.set_tuning(**want)
        ctx._applied_tuning = dict(want)


def clear() -> None:
    with _lock:
        _cache.clear()


def tune(run, npx: int, device: int | None = None, reps: int = 5, warmup: int = 1) -> dict:
    """Tunes the launch shapes on the workload ``run()`` (a callable that
    makes one full library call, e.g. ``lambda: compute_dmsc(img, 0.05)``,
    of ``npx`` total pixels) and caches the result for that size class.
    Returns a report: the choice, the per-candidate median stage times, and
    the whole-call device time (sum of the stages) of the default and of the
    tuned shapes."""
    dev = torch.cuda.current_device() if device is None else device
    ctx = _lib.context(dev)
    limits = ctx.tuning_limits()
    cur = _default_tuning()
    report = {"size_class": size_class(npx), "limits": limits, "stages": {}}

    def measure(stage):
        ctx.set_tuning(**cur)
        for _ in range(warmup):
            run()
        torch.cuda.synchronize()
        ctx.set_profiling(True)
        ts, tot = [], []
        try:
            for _ in range(reps):
                run()
                st = ctx.stage_times()
                ts.append(st[stage] if stage else 0.0)
                tot.append(sum(st.values()))
        finally:
            ctx.set_profiling(False)
        return ts, tot

    _tuning.active = True
    ctx._applied_tuning = None
    try:
        _, tot_default = measure(None)
        for name, stage, gen in TUNABLES:
            timings = {}
            for v in gen(limits):
                cur[name] = v
                timings[v], _ = measure(stage)
            cur[name] = select(timings)
            report["stages"][name] = {str(k): statistics.median(t) for k, t in timings.items()}
        _, tot_tuned = measure(None)
    except Exception:
        ctx.set_tuning(**_default_tuning())
        raise
    finally:
        _tuning.active = False
    with _lock:
        _cache[(dev, size_class(npx))] = dict(cur)
    ctx.set_tuning(**cur)
    ctx._applied_tuning = dict(cur)
    report["choice"] = dict(cur)
    report["default_ms"] = statistics.median(tot_default)
    report["tuned_ms"] = statistics.median(tot_tuned)
    return report
