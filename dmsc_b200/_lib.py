"""ctypes binding of the C ABI in ``include/dmsc_b200.h``.

The product path has no CPU fallback: if ``libdmsc_b200.so`` is missing or no
CUDA device is present, loading raises.
"""

from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdmsc_b200.so")

DUAL, RETURN_GRADIENT, TRACE_RIDGES, TRACE_VALLEYS, TRACE_PEAKS, TRACE_BASINS = 1, 2, 4, 8, 16, 32

# C-ABI exports, in header order (include/dmsc_b200.h).
EXPORTS = (
    "dmsc_b200_create",
    "dmsc_b200_destroy",
    "dmsc_b200_extract",
    "dmsc_b200_fetch",
    "dmsc_b200_set_host_outputs",
    "dmsc_b200_set_host_fetch_outputs",
    "dmsc_b200_set_host_input",
    "dmsc_b200_extract_batch",
    "dmsc_b200_fetch_pair_pixels",
    "dmsc_b200_scatter_pair_grads",
    "dmsc_b200_error_string",
    "dmsc_b200_last_error",
    "dmsc_b200_set_profiling",
    "dmsc_b200_stage_times",
    "dmsc_b200_launch_count",
    "dmsc_b200_loop_counts",
    "dmsc_b200_pairing_timeline",
    "dmsc_b200_set_loop_caps",
    "dmsc_b200_set_tuning",
    "dmsc_b200_get_tuning",
    "dmsc_b200_tuning_limits",
    "dmsc_b200_set_wait_timeout",
    "dmsc_b200_critical_cells_static",
)

STAGES = ("setup", "gradient", "compaction", "saddle_walks", "pairing", "persistence_and_ranks", "survivors",
          "replay", "final_arcs", "label_setup", "labels", "sizes", "fetch_lists", "fetch_geometry")

ERR_TOO_LARGE = 2


class Sizes(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in (
        "max_pts", "min_pts", "sad_pts", "e_max_rows", "e_min_rows", "p_max", "p_min", "ppairs_max", "ppairs_min",
        "grad_indices", "peaks_h", "peaks_w", "ridges", "ridge_offsets", "ridge_arc_offsets", "basins_h", "basins_w",
        "valleys", "valley_offsets", "valley_arc_offsets")]


class Tuning(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("grad_shape", "label_shape", "pair_blocks_per_sm",
                                            "replay_blocks_per_sm", "emit_blocks_per_sm", "seg_cursors",
                                            "pair_shape", "replay_shape", "emit_shape")]


class Outputs(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in (
        "max_pts", "min_pts", "sad_pts", "e_max", "e_min", "p_max", "p_min", "ppairs_max", "ppairs_min", "ridges",
        "ridge_offsets", "ridge_arc_offsets", "valleys", "valley_offsets", "valley_arc_offsets")]


_lib = None
_lock = threading.Lock()


def load():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"dmsc_b200 CUDA library not found at {LIB_PATH}; build it with `python -m dmsc_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        lib.dmsc_b200_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]
        lib.dmsc_b200_create.restype = ctypes.c_int
        lib.dmsc_b200_destroy.argtypes = [ctypes.c_void_p]
        lib.dmsc_b200_destroy.restype = None
        lib.dmsc_b200_extract.argtypes = [
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_uint,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Sizes), ctypes.c_void_p]
        lib.dmsc_b200_extract.restype = ctypes.c_int
        lib.dmsc_b200_fetch.argtypes = [ctypes.c_void_p, ctypes.POINTER(Outputs), ctypes.c_void_p]
        lib.dmsc_b200_fetch.restype = ctypes.c_int
        lib.dmsc_b200_set_host_outputs.argtypes = [ctypes.c_void_p] * 4
        lib.dmsc_b200_set_host_outputs.restype = ctypes.c_int
        lib.dmsc_b200_set_host_input.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.dmsc_b200_set_host_input.restype = ctypes.c_int
        lib.dmsc_b200_set_host_fetch_outputs.argtypes = [ctypes.c_void_p, ctypes.POINTER(Outputs)]
        lib.dmsc_b200_set_host_fetch_outputs.restype = ctypes.c_int
        lib.dmsc_b200_extract_batch.argtypes = [
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
            ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_ubyte), ctypes.c_uint, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Sizes), ctypes.c_void_p]
        lib.dmsc_b200_extract_batch.restype = ctypes.c_int
        lib.dmsc_b200_fetch_pair_pixels.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 5
        lib.dmsc_b200_fetch_pair_pixels.restype = ctypes.c_int
        lib.dmsc_b200_scatter_pair_grads.argtypes = [
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
            ctypes.c_int64, ctypes.c_void_p]
        lib.dmsc_b200_scatter_pair_grads.restype = ctypes.c_int
        lib.dmsc_b200_error_string.argtypes = [ctypes.c_int]
        lib.dmsc_b200_error_string.restype = ctypes.c_char_p
        lib.dmsc_b200_last_error.argtypes = [ctypes.c_void_p]
        lib.dmsc_b200_last_error.restype = ctypes.c_char_p
        lib.dmsc_b200_set_profiling.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.dmsc_b200_set_profiling.restype = ctypes.c_int
        lib.dmsc_b200_stage_times.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int]
        lib.dmsc_b200_stage_times.restype = ctypes.c_int
        lib.dmsc_b200_launch_count.argtypes = [ctypes.c_void_p]
        lib.dmsc_b200_launch_count.restype = ctypes.c_longlong
        lib.dmsc_b200_loop_counts.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        lib.dmsc_b200_loop_counts.restype = ctypes.c_int
        lib.dmsc_b200_pairing_timeline.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
        lib.dmsc_b200_pairing_timeline.restype = ctypes.c_int
        lib.dmsc_b200_set_loop_caps.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.dmsc_b200_set_loop_caps.restype = ctypes.c_int
        lib.dmsc_b200_set_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(Tuning)]
        lib.dmsc_b200_set_tuning.restype = ctypes.c_int
        lib.dmsc_b200_get_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(Tuning)]
        lib.dmsc_b200_get_tuning.restype = ctypes.c_int
        lib.dmsc_b200_tuning_limits.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        lib.dmsc_b200_tuning_limits.restype = ctypes.c_int
        lib.dmsc_b200_set_wait_timeout.argtypes = [ctypes.c_void_p, ctypes.c_double]
        lib.dmsc_b200_set_wait_timeout.restype = ctypes.c_int
        lib.dmsc_b200_critical_cells_static.argtypes = [
            ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.dmsc_b200_critical_cells_static.restype = ctypes.c_int
        _lib = lib
        return lib


class Context:
    """Owns one device workspace (a ``dmsc_b200_context``)."""

    def __init__(self, device: int):
        self.lib = load()
        self.device = device
        h = ctypes.c_void_p()
        rc = self.lib.dmsc_b200_create(ctypes.byref(h), device)
        if rc != 0:
            raise RuntimeError(f"dmsc_b200_create failed on cuda:{device}: {self.lib.dmsc_b200_error_string(rc).decode()}")
        self.h = h

    def check(self, rc: int, what: str):
        if rc == 0:
            return
        msg = self.lib.dmsc_b200_last_error(self.h).decode() or self.lib.dmsc_b200_error_string(rc).decode()
        raise RuntimeError(f"{what}: {msg}")

    def set_profiling(self, on: bool):
        self.check(self.lib.dmsc_b200_set_profiling(self.h, 1 if on else 0), "dmsc_b200_set_profiling")

    def stage_times(self) -> dict:
        buf = (ctypes.c_float * 32)()
        n = self.lib.dmsc_b200_stage_times(self.h, buf, 32)
        if n < 0:
            raise RuntimeError("stage times unavailable (profiling off or no call)")
        return {STAGES[k]: float(buf[k]) for k in range(min(n, len(STAGES)))}

    def launch_count(self) -> int:
        return int(self.lib.dmsc_b200_launch_count(self.h))

    def loop_counts(self) -> dict:
        buf = (ctypes.c_int * 6)()
        n = self.lib.dmsc_b200_loop_counts(self.h, buf, 6)
        names = ("pair_rounds_faces", "pair_rounds_vertices", "replay_rounds_faces", "replay_rounds_vertices",
                 "emit_levels_faces", "emit_levels_vertices")
        return {names[k]: int(buf[k]) for k in range(max(n, 0))}

    def set_loop_caps(self, pair_rounds: int = 0, replay_rounds: int = 0, emit_levels: int = 0):
        """Lowers the device loop bounds of the following calls (0 = normal)."""
        self.check(self.lib.dmsc_b200_set_loop_caps(self.h, pair_rounds, replay_rounds, emit_levels),
                   "dmsc_b200_set_loop_caps")

    def set_tuning(self, **kw):
        t = self.get_tuning()
        for k, v in kw.items():
            setattr(t, k, int(v))
        self.check(self.lib.dmsc_b200_set_tuning(self.h, ctypes.byref(t)), "dmsc_b200_set_tuning")

    def get_tuning(self) -> Tuning:
        t = Tuning()
        self.check(self.lib.dmsc_b200_get_tuning(self.h, ctypes.byref(t)), "dmsc_b200_get_tuning")
        return t

    def tuning_limits(self) -> dict:
        buf = (ctypes.c_int * 9)()
        if self.lib.dmsc_b200_tuning_limits(self.h, buf, 9) != 9:
            raise RuntimeError("dmsc_b200_tuning_limits failed")
        return dict(zip(("grad_shapes", "label_shapes", "pair_blocks_per_sm", "replay_blocks_per_sm",
                         "emit_blocks_per_sm", "seg_cursors", "pair_shapes", "replay_shapes", "emit_shapes"),
                        list(buf)))

    def set_wait_timeout(self, seconds: float):
        self.check(self.lib.dmsc_b200_set_wait_timeout(self.h, float(seconds)), "dmsc_b200_set_wait_timeout")

    def timelines(self, counts: bool = False) -> dict:
        """Per-round / per-level durations (us) of the device loops of the last
        call; with ``counts``, (durations, items per round) per loop."""
        buf = (ctypes.c_longlong * 896)()
        if self.lib.dmsc_b200_pairing_timeline(self.h, buf, 896) < 0:
            return {}
        out = {}
        for blk, name in enumerate(("pairing_faces", "pairing_vertices", "emit_faces", "emit_vertices",
                                    "replay_faces", "replay_vertices")):
            t = [x for x in (buf[blk * 64 + k] for k in range(64)) if x > 0]
            d = tuple((b - a) / 1000.0 for a, b in zip(t, t[1:]))
            out[name] = (d, tuple(buf[384 + blk * 64 + k] for k in range(len(t)))) if counts else d
            if counts and blk < 2:  # pairing: phase A part of each round (us)
                out[name + "_phase_a"] = (tuple((buf[768 + blk * 64 + k] - t[k]) / 1000.0
                                                for k in range(len(t) - 1) if buf[768 + blk * 64 + k] > 0), ())
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.dmsc_b200_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_tls = threading.local()


def context(device: int) -> Context:
    """Per-thread, per-device context (a context is not thread-safe)."""
    ctxs = getattr(_tls, "ctxs", None)
    if ctxs is None:
        ctxs = _tls.ctxs = {}
    c = ctxs.get(device)
    if c is None:
        c = ctxs[device] = Context(device)
    return c
