"""ctypes front end of the C restatement in ``oracle/dmsc_oracle.c``.

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` are the only callers, always as the checker.

``run(img, thr, ...)`` mirrors the reference native entry
``dmsc_cpu.extract_dmsc(scalar_field, persistence_threshold, return_gradient,
is_dual, trace_max_arcs, trace_min_arcs, trace_max_groups, trace_min_groups)``
(dmsc/csrc/dmsc_cpu.cpp:53-107, 177-181) and returns the same 19 tensors in the
same order, plus a dict of internal stages for kernel-level comparisons.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "dmsc_oracle.c")
LIB = os.path.join(HERE, "liboracle.so")

FIELDS = (
    "shape max_pts min_pts sad_pts e_max e_min p_max p_min ppairs_max ppairs_min grad_indices "
    "peaks ridges ridge_offsets ridge_arc_offsets basins valleys valley_offsets valley_arc_offsets"
).split()
DEBUG_FIELDS = (
    "paired_with crit_mins crit_saddles crit_maxes saddle_values saddle_order_desc "
    "pair_min pers_min pair_max pers_max min_alive max_alive uf_min uf_max "
    "replay_parent_min replay_parent_max ev_min ev_max raw_arcs cancels_min cancels_max min_vals max_vals"
).split()

FL_DUAL, FL_GRAD, FL_RIDGES, FL_VALLEYS, FL_PEAKS, FL_BASINS = 1, 2, 4, 8, 16, 32

_lib = None


def build(force: bool = False) -> str:
    """Compile the C oracle into ``oracle/liboracle.so`` (gcc, -O2)."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", "-O2", "-std=c11", "-shared", "-fPIC", "-o", LIB, SRC, "-lm"])
    return LIB


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(LIB)
        lib.dmsc_oracle_run.restype = ctypes.c_void_p
        lib.dmsc_oracle_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int]
        lib.dmsc_oracle_field.argtypes = [
            ctypes.c_void_p,
            ctypes.c_int,
            ctypes.POINTER(ctypes.c_void_p),
            ctypes.POINTER(ctypes.c_int64),
            ctypes.POINTER(ctypes.c_int64),
            ctypes.POINTER(ctypes.c_int),
            ctypes.POINTER(ctypes.c_int),
        ]
        lib.dmsc_oracle_status.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
        lib.dmsc_oracle_free.argtypes = [ctypes.c_void_p]
        _lib = lib
    return _lib


def flags_of(is_dual=False, return_gradient=False, trace_max_arcs=False, trace_min_arcs=False,
             trace_max_groups=False, trace_min_groups=False) -> int:
    f = 0
    f |= FL_DUAL if is_dual else 0
    f |= FL_GRAD if return_gradient else 0
    f |= FL_RIDGES if trace_max_arcs else 0
    f |= FL_VALLEYS if trace_min_arcs else 0
    f |= FL_PEAKS if trace_max_groups else 0
    f |= FL_BASINS if trace_min_groups else 0
    return f


def run(img, persistence_threshold, return_gradient=False, is_dual=False, trace_max_arcs=False,
        trace_min_arcs=False, trace_max_groups=False, trace_min_groups=False, debug=False):
    """One 2-D field through the C oracle. Returns a 19-tuple of CPU tensors
    (and a dict of internal stages when ``debug``)."""
    lib = _load()
    a = np.ascontiguousarray(torch.as_tensor(img).detach().cpu().numpy(), dtype=np.float32)
    assert a.ndim == 2
    H, W = a.shape
    flags = flags_of(is_dual, return_gradient, trace_max_arcs, trace_min_arcs, trace_max_groups, trace_min_groups)
    h = lib.dmsc_oracle_run(a.ctypes.data, H, W, ctypes.c_float(persistence_threshold), flags)
    try:
        msg = ctypes.create_string_buffer(256)
        st = lib.dmsc_oracle_status(h, msg, 256)
        if st != 0:
            raise RuntimeError(msg.value.decode())
        out = []
        n = len(FIELDS) + (len(DEBUG_FIELDS) if debug else 0)
        for k in range(n):
            p = ctypes.c_void_p()
            d0, d1 = ctypes.c_int64(), ctypes.c_int64()
            nd, isf = ctypes.c_int(), ctypes.c_int()
            lib.dmsc_oracle_field(h, k, ctypes.byref(p), ctypes.byref(d0), ctypes.byref(d1), ctypes.byref(nd),
                                  ctypes.byref(isf))
            shape = (d0.value,) if nd.value == 1 else (d0.value, d1.value)
            cnt = int(np.prod(shape))
            ctype = ctypes.c_float if isf.value else ctypes.c_int32
            if cnt > 0:
                buf = (ctype * cnt).from_address(p.value)
                arr = np.frombuffer(buf, dtype=np.float32 if isf.value else np.int32, count=cnt).copy()
            else:
                arr = np.empty(0, dtype=np.float32 if isf.value else np.int32)
            out.append(torch.from_numpy(arr.reshape(shape)))
    finally:
        lib.dmsc_oracle_free(h)
    main = tuple(out[: len(FIELDS)])
    if debug:
        return main, dict(zip(DEBUG_FIELDS, out[len(FIELDS):]))
    return main


def compute_dmsc(img, persistence_threshold, return_gradient=True, is_dual=False, trace_valleys=True,
                 trace_ridges=True, trace_peaks=True, trace_basins=True):
    """Oracle twin of ``dmsc.compute_dmsc`` (dmsc/dmsc.py:230-276) for 2-D or 3-D CPU input."""
    img = torch.as_tensor(img)
    kw = dict(return_gradient=return_gradient, is_dual=is_dual, trace_max_arcs=trace_ridges,
              trace_min_arcs=trace_valleys, trace_max_groups=trace_peaks, trace_min_groups=trace_basins)
    if img.dim() == 2:
        return run(img, persistence_threshold, **kw)
    return [run(x, persistence_threshold, **kw) for x in img]
