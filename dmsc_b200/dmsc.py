"""Drop-in mirror of the reference Python API (dmsc/dmsc.py:1-276).

``compute_dmsc`` keeps the reference signature, argument meaning, error types
and the 19-field ``MSComplex`` result; the computation runs on the GPU through
the C ABI (include/dmsc_b200.h). CUDA input stays on its device; CPU input is
copied to the current CUDA device and the results are returned on the CPU,
which is the reference's device contract for CPU tensors. There is no CPU
compute path.
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, fields

import torch

from . import _lib


@dataclass
class MSComplex:
    """The extracted Morse-Smale complex (field order of dmsc/dmsc.py:49-70).

    Grid mapping by ``is_dual``: primal maxima are faces ((H+1) x (W+1) pixel
    corners) and minima vertices (pixels); the dual swaps them. Geometry is
    raw cell ids, ``cell = type + 4 * (y * (W+1) + x)``.
    """

    shape: torch.Tensor

    max_pts: torch.Tensor
    min_pts: torch.Tensor
    sad_pts: torch.Tensor
    e_max: torch.Tensor
    e_min: torch.Tensor
    p_max: torch.Tensor
    p_min: torch.Tensor
    ppairs_max: torch.Tensor
    ppairs_min: torch.Tensor
    grad_indices: torch.Tensor

    peaks: torch.Tensor
    ridges: torch.Tensor
    ridge_offsets: torch.Tensor
    ridge_arc_offsets: torch.Tensor

    basins: torch.Tensor
    valleys: torch.Tensor
    valley_offsets: torch.Tensor
    valley_arc_offsets: torch.Tensor

    def __str__(self):
        output = "MSComplex("
        for field in fields(self):
            value = getattr(self, field.name)
            if hasattr(value, "shape"):
                output += f" {field.name}:{tuple(value.shape)},"
        return output + ")"

    @property
    def Nx(self) -> int:
        return int(self.shape[1].item()) + 1

    def to_coordinates_yx(self, cell_tensor: torch.Tensor, staggered: bool = True) -> torch.Tensor:
        """Decodes cell ids into [y, x] (dmsc/dmsc.py:87-118); with ``staggered``
        edges and corners get their -0.5 sub-pixel offsets."""
        if cell_tensor.numel() == 0:
            dtype = torch.float32 if staggered else torch.int32
            return torch.empty((0, 2), dtype=dtype, device=cell_tensor.device)
        c_type = cell_tensor % 4
        idx = cell_tensor // 4
        y = idx // self.Nx
        x = idx % self.Nx
        if not staggered:
            return torch.stack([y, x], dim=-1).to(torch.int32)
        y = y.float()
        x = x.float()
        y -= torch.where((c_type == 2) | (c_type == 3), 0.5, 0.0)
        x -= torch.where((c_type == 1) | (c_type == 3), 0.5, 0.0)
        return torch.stack([y, x], dim=-1)

    @property
    def offset_max_pts_yx(self):
        return self.to_coordinates_yx(self.max_pts)

    @property
    def offset_min_pts_yx(self):
        return self.to_coordinates_yx(self.min_pts)

    @property
    def offset_sad_pts_yx(self):
        return self.to_coordinates_yx(self.sad_pts)

    def get_ridge(self, saddle_idx: int, split_arcs=False):
        """CSR slice of one saddle's ridge (dmsc/dmsc.py:132-143)."""
        start = self.ridge_offsets[saddle_idx]
        end = self.ridge_offsets[saddle_idx + 1] if saddle_idx + 1 < len(self.ridge_offsets) else len(self.ridges)
        pts = self.ridges[start:end]
        if split_arcs:
            split = self.ridge_arc_offsets[saddle_idx]
            return pts[: split - start], pts[split - start: end - start]
        return pts

    def get_valley(self, saddle_idx: int, split_arcs=False):
        """CSR slice of one saddle's valley (dmsc/dmsc.py:145-156)."""
        start = self.valley_offsets[saddle_idx]
        end = self.valley_offsets[saddle_idx + 1] if saddle_idx + 1 < len(self.valley_offsets) else len(self.valleys)
        pts = self.valleys[start:end]
        if split_arcs:
            split = self.valley_arc_offsets[saddle_idx]
            return pts[: split - start], pts[split - start: end - start]
        return pts

    def __iter__(self):
        # The 19 tensors in field order, as the reference's astuple-based
        # iteration yields them (dmsc/dmsc.py:158-159), without its deep copies.
        return iter(tuple(getattr(self, f.name) for f in fields(self)))

    def __len__(self):
        return 19

    def __getitem__(self, i):
        return getattr(self, fields(self)[i].name)

    def _no_plots(self, *a, **k):
        raise NotImplementedError("visualisation (matplotlib dashboards) is not part of dmsc_b200")

    plot = plot_gradient = plot_complex = plot_barcode = _no_plots


def _validate(img):
    """Error contract of dmsc/dmsc.py:245-254."""
    if img.dim() not in (2, 3):
        raise ValueError(f"Input tensor must be 2D [H, W] or 3D [B, H, W]. Got {img.dim()}D.")
    if img.layout != torch.strided:
        raise ValueError(f"Input tensor must use strided layout. Got {img.layout}.")
    if img.dtype != torch.float32:
        raise TypeError(f"Input tensor must have dtype torch.float32. Got {img.dtype}.")
    if img.dim() == 3 and img.shape[0] == 0:
        raise ValueError("Batch dimension must be non-empty.")
    if img.shape[-2] == 0 or img.shape[-1] == 0:
        raise ValueError(f"Spatial dimensions must be non-empty. Got {tuple(img.shape[-2:])}.")


def _flags(return_gradient, is_dual, trace_ridges, trace_valleys, trace_peaks, trace_basins) -> int:
    f = 0
    f |= _lib.DUAL if is_dual else 0
    f |= _lib.RETURN_GRADIENT if return_gradient else 0
    f |= _lib.TRACE_RIDGES if trace_ridges else 0
    f |= _lib.TRACE_VALLEYS if trace_valleys else 0
    f |= _lib.TRACE_PEAKS if trace_peaks else 0
    f |= _lib.TRACE_BASINS if trace_basins else 0
    return f


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else ctypes.c_void_p(0)


def extract_single(img: torch.Tensor, persistence_threshold: float, flags: int, stream=None) -> tuple:
    """One contiguous float32 [H, W] CUDA image through both C-ABI phases;
    returns the 19 output tensors on the image's device (shape on the CPU)."""
    H, W = int(img.shape[0]), int(img.shape[1])
    dev = img.device
    ctx = _lib.context(dev.index if dev.index is not None else torch.cuda.current_device())
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    i32 = dict(dtype=torch.int32, device=dev)
    dual = bool(flags & _lib.DUAL)
    nidx = (H + 1) * (W + 1)
    grad = torch.empty(4 * nidx, **i32) if flags & _lib.RETURN_GRADIENT else None
    peaks = torch.empty((H, W) if dual else (H + 1, W + 1), **i32) if flags & _lib.TRACE_PEAKS else None
    basins = torch.empty((H + 1, W + 1) if dual else (H, W), **i32) if flags & _lib.TRACE_BASINS else None
    sz = _lib.Sizes()
    rc = ctx.lib.dmsc_b200_extract(ctx.h, ctypes.c_void_p(img.data_ptr()), H, W, ctypes.c_float(persistence_threshold),
                                   flags, _ptr(grad), _ptr(peaks), _ptr(basins), ctypes.byref(sz),
                                   ctypes.c_void_p(s.cuda_stream))
    if rc == _lib.ERR_TOO_LARGE:
        raise RuntimeError(f"Input is too large for 32-bit cell IDs: {H}x{W}")
    ctx.check(rc, "dmsc_b200_extract")
    out = dict(
        max_pts=torch.empty(sz.max_pts, **i32), min_pts=torch.empty(sz.min_pts, **i32),
        sad_pts=torch.empty(sz.sad_pts, **i32), e_max=torch.empty((sz.e_max_rows, 2), **i32),
        e_min=torch.empty((sz.e_min_rows, 2), **i32), p_max=torch.empty(sz.p_max, dtype=torch.float32, device=dev),
        p_min=torch.empty(sz.p_min, dtype=torch.float32, device=dev), ppairs_max=torch.empty(sz.ppairs_max, **i32),
        ppairs_min=torch.empty(sz.ppairs_min, **i32), ridges=torch.empty(sz.ridges, **i32),
        ridge_offsets=torch.empty(sz.ridge_offsets, **i32), ridge_arc_offsets=torch.empty(sz.ridge_arc_offsets, **i32),
        valleys=torch.empty(sz.valleys, **i32), valley_offsets=torch.empty(sz.valley_offsets, **i32),
        valley_arc_offsets=torch.empty(sz.valley_arc_offsets, **i32))
    o = _lib.Outputs(**{k: _ptr(v) for k, v in out.items()})
    ctx.check(ctx.lib.dmsc_b200_fetch(ctx.h, ctypes.byref(o), ctypes.c_void_p(s.cuda_stream)), "dmsc_b200_fetch")
    empty = torch.empty(0, **i32)
    empty2 = torch.empty((0, 0), **i32)
    shape = torch.tensor([H, W], dtype=torch.int32)
    return (shape, out["max_pts"], out["min_pts"], out["sad_pts"], out["e_max"], out["e_min"], out["p_max"],
            out["p_min"], out["ppairs_max"], out["ppairs_min"], grad if grad is not None else empty,
            peaks if peaks is not None else empty2, out["ridges"], out["ridge_offsets"], out["ridge_arc_offsets"],
            basins if basins is not None else empty2, out["valleys"], out["valley_offsets"],
            out["valley_arc_offsets"])


def extract_dmsc(scalar_field, persistence_threshold, return_gradient=False, is_dual=False, trace_max_arcs=False,
                 trace_min_arcs=False, trace_max_groups=False, trace_min_groups=False):
    """Mirror of the reference native entry ``dmsc_gpu.extract_dmsc``
    (dmsc/csrc/dmsc_gpu.cpp:128-180, 249-253): 19-tuple for 2-D input, a list
    of 19-tuples for a 3-D batch (one image after another)."""
    if scalar_field.dim() not in (2, 3) or scalar_field.dtype != torch.float32 or scalar_field.numel() == 0:
        raise RuntimeError("Input tensor must be a non-empty float32 2D [H, W] or 3D [B, H, W] tensor")
    H, W = int(scalar_field.shape[-2]), int(scalar_field.shape[-1])
    if H + 1 > (2**31 - 1) // 4 // (W + 1):  # input_validation.hxx:24-26
        raise RuntimeError(f"Input is too large for 32-bit cell IDs: {H}x{W}")
    if not torch.cuda.is_available():
        raise RuntimeError("dmsc_b200 requires a CUDA device; there is no CPU compute path")
    on_cpu = scalar_field.device.type != "cuda"
    flags = _flags(return_gradient, is_dual, trace_max_arcs, trace_min_arcs, trace_max_groups, trace_min_groups)
    if on_cpu:
        x = scalar_field.contiguous().to("cuda", non_blocking=True)
    else:
        x = scalar_field.contiguous()
    with torch.cuda.device(x.device):
        if x.dim() == 2:
            res = extract_single(x, persistence_threshold, flags)
            return _to_host(res) if on_cpu else res
        outs = [extract_single(x[b], persistence_threshold, flags) for b in range(x.shape[0])]
        return [_to_host(r) for r in outs] if on_cpu else outs


def _to_host(res: tuple) -> tuple:
    """Device outputs -> CPU tensors for a CPU caller: asynchronous copies into
    pinned (cached) host buffers on the current stream, one synchronisation."""
    out = []
    for t in res:
        if t.device.type == "cpu":
            out.append(t)
            continue
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        if t.numel():
            h.copy_(t, non_blocking=True)
        out.append(h)
    torch.cuda.current_stream().synchronize()
    return tuple(out)


def compute_dmsc(img, persistence_threshold, return_gradient=True, is_dual=False, trace_valleys=True,
                 trace_ridges=True, trace_peaks=True, trace_basins=True, verbose=False):
    """Extracts the discrete Morse-Smale complex (dmsc/dmsc.py:230-276).

    Returns one ``MSComplex`` for a 2-D [H, W] float32 tensor or a list of
    them for a 3-D [B, H, W] batch.
    """
    _validate(img)
    start = time.perf_counter()
    output = extract_dmsc(img, persistence_threshold, return_gradient, is_dual, trace_max_arcs=trace_ridges,
                          trace_min_arcs=trace_valleys, trace_max_groups=trace_peaks, trace_min_groups=trace_basins)
    if verbose:
        print(f"Time for MS-complex computation: {(time.perf_counter() - start) * 1000:.3f} ms")
    if img.dim() == 2:
        return MSComplex(*output)
    return [MSComplex(*res) for res in output]
