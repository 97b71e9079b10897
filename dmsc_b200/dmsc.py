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

from . import _lib, tuning


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

    # Host copies of the CSR offsets, read from the device once on first use
    # (one transfer per array instead of one synchronisation per slice).
    def _host_offsets(self, name: str) -> list:
        cache = self.__dict__.setdefault("_host_cache", {})
        if name not in cache:
            cache[name] = getattr(self, name).tolist()
        return cache[name]

    def _arc(self, pts_name: str, off_name: str, aoff_name: str, saddle_idx: int, split_arcs: bool):
        off = self._host_offsets(off_name)
        pts = getattr(self, pts_name)
        saddle_idx = int(saddle_idx)
        start = off[saddle_idx]
        end = off[saddle_idx + 1] if saddle_idx + 1 < len(off) else len(pts)
        seg = pts[start:end]
        if split_arcs:
            split = self._host_offsets(aoff_name)[saddle_idx]
            return seg[: split - start], seg[split - start: end - start]
        return seg

    def get_ridge(self, saddle_idx: int, split_arcs=False):
        """CSR slice of one saddle's ridge (dmsc/dmsc.py:132-143): the same
        slices, as views of ``ridges``; the offsets are read once per complex,
        so slicing does not synchronise with the device."""
        return self._arc("ridges", "ridge_offsets", "ridge_arc_offsets", saddle_idx, split_arcs)

    def get_valley(self, saddle_idx: int, split_arcs=False):
        """CSR slice of one saddle's valley (dmsc/dmsc.py:145-156); see get_ridge."""
        return self._arc("valleys", "valley_offsets", "valley_arc_offsets", saddle_idx, split_arcs)

    def _arcs(self, pts_name: str, off_name: str, aoff_name: str, saddle_idx):
        pts, off, aoff = getattr(self, pts_name), getattr(self, off_name), getattr(self, aoff_name)
        idx = torch.as_tensor(saddle_idx, dtype=torch.int64, device=off.device).reshape(-1)
        n = len(off) - 1
        if idx.numel() and n > 0:
            idx = torch.where(idx < 0, idx + n, idx)
        start = off[idx].to(torch.int64)
        length = off[idx + 1].to(torch.int64) - start
        new_off = torch.zeros(idx.numel() + 1, dtype=torch.int64, device=off.device)
        torch.cumsum(length, 0, out=new_off[1:])
        hl = self._host_offsets(off_name)
        total = int(sum(hl[i + 1] - hl[i] for i in idx.tolist())) if idx.numel() else 0
        # position of every output cell in `pts`: its arc's start + rank inside the arc
        seg = torch.repeat_interleave(torch.arange(idx.numel(), device=off.device), length, output_size=total)
        pos = start[seg] + torch.arange(total, device=off.device) - new_off[:-1][seg]
        cells = pts[pos]
        first = (aoff[idx].to(torch.int64) - start) + new_off[:-1]
        return cells, new_off.to(torch.int32), first.to(torch.int32)

    def get_ridges(self, saddle_idx):
        """Ridges of many saddles at once (batched form of get_ridge):
        ``(cells, offsets, arc_offsets)`` in CSR layout over the given saddle
        indices, with ``cells[offsets[k]:offsets[k+1]] == get_ridge(i_k)`` and
        ``arc_offsets[k]`` the end of its first arc. One gather on the
        device."""
        return self._arcs("ridges", "ridge_offsets", "ridge_arc_offsets", saddle_idx)

    def get_valleys(self, saddle_idx):
        """Valleys of many saddles at once (batched form of get_valley)."""
        return self._arcs("valleys", "valley_offsets", "valley_arc_offsets", saddle_idx)

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


def _host_like(t):
    """Pinned host tensor shaped like ``t`` (None stays None)."""
    return None if t is None else torch.empty(t.shape, dtype=t.dtype, pin_memory=True)


def extract_single(img: torch.Tensor, persistence_threshold: float, flags: int, stream=None,
                   host_fixed: bool = False, host_src: torch.Tensor | None = None) -> tuple:
    """One contiguous float32 [H, W] CUDA image through both C-ABI phases;
    returns the 19 output tensors on the image's device (shape on the CPU).
    With ``host_fixed`` the gradient and label maps are returned in pinned
    host tensors that the library fills while the rest of the call runs
    (``dmsc_b200_set_host_outputs``); they are complete once the stream has
    passed the call. With ``host_src`` (a pinned host copy of the image)
    ``img`` is only the device destination: the library uploads the image
    itself, overlapped with the gradient (``dmsc_b200_set_host_input``);
    ``host_src`` must stay unchanged until the stream has passed the call."""
    H, W = int(img.shape[0]), int(img.shape[1])
    dev = img.device
    ctx = _lib.context(dev.index if dev.index is not None else torch.cuda.current_device())
    tuning.apply(ctx, H * W)
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    i32 = dict(dtype=torch.int32, device=dev)
    dual = bool(flags & _lib.DUAL)
    nidx = (H + 1) * (W + 1)
    grad = torch.empty(4 * nidx, **i32) if flags & _lib.RETURN_GRADIENT else None
    peaks = torch.empty((H, W) if dual else (H + 1, W + 1), **i32) if flags & _lib.TRACE_PEAKS else None
    basins = torch.empty((H + 1, W + 1) if dual else (H, W), **i32) if flags & _lib.TRACE_BASINS else None
    if host_fixed:
        hg, hp, hb = _host_like(grad), _host_like(peaks), _host_like(basins)
        ctx.check(ctx.lib.dmsc_b200_set_host_outputs(ctx.h, _ptr(hg), _ptr(hp), _ptr(hb)),
                  "dmsc_b200_set_host_outputs")
    if host_src is not None:
        ctx.check(ctx.lib.dmsc_b200_set_host_input(ctx.h, _ptr(host_src)), "dmsc_b200_set_host_input")
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
    if host_fixed:  # variable outputs copied to pinned host memory as the fetch writes them
        hout = {k: _host_like(v) for k, v in out.items()}
        ho = _lib.Outputs(**{k: _ptr(v) for k, v in hout.items()})
        ctx.check(ctx.lib.dmsc_b200_set_host_fetch_outputs(ctx.h, ctypes.byref(ho)), "dmsc_b200_set_host_fetch_outputs")
    ctx.check(ctx.lib.dmsc_b200_fetch(ctx.h, ctypes.byref(o), ctypes.c_void_p(s.cuda_stream)), "dmsc_b200_fetch")
    empty = torch.empty(0, **i32)
    empty2 = torch.empty((0, 0), **i32)
    shape = torch.tensor([H, W], dtype=torch.int32)
    if host_fixed:  # host tensors, complete once the stream has passed the fetch
        grad, peaks, basins = hg, hp, hb
        out = hout
        empty = torch.empty(0, dtype=torch.int32)
        empty2 = torch.empty((0, 0), dtype=torch.int32)
    return (shape, out["max_pts"], out["min_pts"], out["sad_pts"], out["e_max"], out["e_min"], out["p_max"],
            out["p_min"], out["ppairs_max"], out["ppairs_min"], grad if grad is not None else empty,
            peaks if peaks is not None else empty2, out["ridges"], out["ridge_offsets"], out["ridge_arc_offsets"],
            basins if basins is not None else empty2, out["valleys"], out["valley_offsets"],
            out["valley_arc_offsets"])


# Indices (H+1)*(W+1) summed over the images of one device batch. The library
# takes up to 2^29 - 1 (int32 cell ids over the batch); 2^28 keeps one device
# batch's workspace to a few tens of GB of HBM.
BATCH_INDEX_CAP = 1 << 28

_FIELDS = ("max_pts", "min_pts", "sad_pts", "e_max", "e_min", "p_max", "p_min", "ppairs_max", "ppairs_min", "ridges",
           "ridge_offsets", "ridge_arc_offsets", "valleys", "valley_offsets", "valley_arc_offsets")
_SIZE_OF = dict(max_pts="max_pts", min_pts="min_pts", sad_pts="sad_pts", e_max="e_max_rows", e_min="e_min_rows",
                p_max="p_max", p_min="p_min", ppairs_max="ppairs_max", ppairs_min="ppairs_min", ridges="ridges",
                ridge_offsets="ridge_offsets", ridge_arc_offsets="ridge_arc_offsets", valleys="valleys",
                valley_offsets="valley_offsets", valley_arc_offsets="valley_arc_offsets")


def _batch_raw(images, thresholds, is_dual, flags: int, stream=None, flat=None, pair_pixels=False, host_fixed=False):
    """Both C-ABI phases of one device batch. Returns the batch-wide output
    tensors (``out``, field -> tensor, images back to back), the per-image
    lengths of each (``lens``), the image shapes and orientations and the
    stream. ``flat`` may hold the images already back to back; with
    ``pair_pixels`` the pixel pairs of every p_max / p_min entry are fetched
    too (``plus_max``, ``minus_max``, ``plus_min``, ``minus_min``)."""
    B = len(images)
    dev = images[0].device
    ctx = _lib.context(dev.index if dev.index is not None else torch.cuda.current_device())
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    i32 = dict(dtype=torch.int32, device=dev)
    Hs = [int(x.shape[0]) for x in images]
    Ws = [int(x.shape[1]) for x in images]
    duals = [bool(d) for d in is_dual]
    if flat is None:
        flat = images[0].reshape(-1) if B == 1 else torch.cat([x.reshape(-1) for x in images])
    nidx = [(h + 1) * (w + 1) for h, w in zip(Hs, Ws)]
    npx = [h * w for h, w in zip(Hs, Ws)]
    tuning.apply(ctx, sum(npx))
    pk_n = [p if d else n for p, n, d in zip(npx, nidx, duals)]
    bs_n = [n if d else p for p, n, d in zip(npx, nidx, duals)]
    grad = torch.empty(4 * sum(nidx), **i32) if flags & _lib.RETURN_GRADIENT else None
    peaks = torch.empty(sum(pk_n), **i32) if flags & _lib.TRACE_PEAKS else None
    basins = torch.empty(sum(bs_n), **i32) if flags & _lib.TRACE_BASINS else None
    if host_fixed:  # gradient and labels copied to pinned host memory while the call runs
        hg, hp, hb = _host_like(grad), _host_like(peaks), _host_like(basins)
        ctx.check(ctx.lib.dmsc_b200_set_host_outputs(ctx.h, _ptr(hg), _ptr(hp), _ptr(hb)),
                  "dmsc_b200_set_host_outputs")
    sz = (_lib.Sizes * B)()
    rc = ctx.lib.dmsc_b200_extract_batch(
        ctx.h, ctypes.c_void_p(flat.data_ptr()), B, (ctypes.c_int * B)(*Hs), (ctypes.c_int * B)(*Ws),
        (ctypes.c_float * B)(*[float(t) for t in thresholds]), (ctypes.c_ubyte * B)(*[int(d) for d in duals]), flags,
        _ptr(grad), _ptr(peaks), _ptr(basins), sz, ctypes.c_void_p(s.cuda_stream))
    if rc == _lib.ERR_TOO_LARGE and B == 1:
        raise RuntimeError(f"Input is too large for 32-bit cell IDs: {Hs[0]}x{Ws[0]}")
    ctx.check(rc, "dmsc_b200_extract_batch")
    lens = {f: [int(getattr(sz[b], _SIZE_OF[f])) for b in range(B)] for f in _FIELDS}
    out = {}
    for f in _FIELDS:
        n = sum(lens[f])
        dt = torch.float32 if f in ("p_max", "p_min") else torch.int32
        out[f] = torch.empty((n, 2) if f in ("e_max", "e_min") else n, dtype=dt, device=dev)
    o = _lib.Outputs(**{k: _ptr(v) for k, v in out.items()})
    if host_fixed:  # variable outputs copied to pinned host memory as the fetch writes them
        hout = {k: _host_like(v) for k, v in out.items()}
        ho = _lib.Outputs(**{k: _ptr(v) for k, v in hout.items()})
        ctx.check(ctx.lib.dmsc_b200_set_host_fetch_outputs(ctx.h, ctypes.byref(ho)), "dmsc_b200_set_host_fetch_outputs")
    ctx.check(ctx.lib.dmsc_b200_fetch(ctx.h, ctypes.byref(o), ctypes.c_void_p(s.cuda_stream)), "dmsc_b200_fetch")
    if host_fixed:
        out = hout
    if pair_pixels:
        for f in ("plus_max", "minus_max", "plus_min", "minus_min"):
            side = f.split("_")[1]
            out[f] = torch.empty(out["p_" + side].numel(), **i32)
            lens[f] = lens["p_" + side]
        ctx.check(ctx.lib.dmsc_b200_fetch_pair_pixels(
            ctx.h, _ptr(out["plus_max"]), _ptr(out["minus_max"]), _ptr(out["plus_min"]), _ptr(out["minus_min"]),
            ctypes.c_void_p(s.cuda_stream)), "dmsc_b200_fetch_pair_pixels")
    if host_fixed:
        grad, peaks, basins = hg, hp, hb
    if grad is not None:
        out["grad_indices"] = grad
        lens["grad_indices"] = [4 * n for n in nidx]
    if peaks is not None:
        out["peaks"] = peaks
        lens["peaks"] = pk_n
    if basins is not None:
        out["basins"] = basins
        lens["basins"] = bs_n
    return out, lens, Hs, Ws, duals, s


def extract_batch(images, thresholds, is_dual, flags: int, to_host: bool = False, stream=None) -> list:
    """Contiguous float32 2-D CUDA images of any sizes (one device), each with
    its own threshold and orientation, through one batched extract and one
    fetch (``dmsc_b200_extract_batch``). Returns one 19-tuple per image; each
    tensor is a view of one batch-wide output tensor (on the CPU when
    ``to_host``). ``flags``' DUAL bit is ignored in favour of ``is_dual``."""
    B = len(images)
    dev = images[0].device
    out, lens, Hs, Ws, duals, s = _batch_raw(images, thresholds, is_dual, flags, stream, host_fixed=to_host)
    grad, peaks, basins = out.get("grad_indices"), out.get("peaks"), out.get("basins")
    if to_host:
        with torch.cuda.stream(s):
            out = dict(zip(out.keys(), _to_host(tuple(out.values()))))
    parts = {k: torch.split(v, lens[k]) for k, v in out.items()}
    odev = torch.device("cpu") if to_host else dev
    empty = torch.empty(0, dtype=torch.int32, device=odev)
    empty2 = torch.empty((0, 0), dtype=torch.int32, device=odev)
    res = []
    for b in range(B):
        H, W, d = Hs[b], Ws[b], duals[b]
        g = parts["grad_indices"][b] if grad is not None else empty
        pk = parts["peaks"][b].view((H, W) if d else (H + 1, W + 1)) if peaks is not None else empty2
        bs = parts["basins"][b].view((H + 1, W + 1) if d else (H, W)) if basins is not None else empty2
        q = {f: parts[f][b] for f in _FIELDS}
        res.append((torch.tensor([H, W], dtype=torch.int32), q["max_pts"], q["min_pts"], q["sad_pts"], q["e_max"],
                    q["e_min"], q["p_max"], q["p_min"], q["ppairs_max"], q["ppairs_min"], g, pk, q["ridges"],
                    q["ridge_offsets"], q["ridge_arc_offsets"], bs, q["valleys"], q["valley_offsets"],
                    q["valley_arc_offsets"]))
    return res


def _chunks(shapes):
    """Consecutive image ranges whose index counts fit one device batch."""
    start, acc = 0, 0
    for b, (h, w) in enumerate(shapes):
        n = (h + 1) * (w + 1)
        if b > start and acc + n > BATCH_INDEX_CAP:
            yield start, b
            start, acc = b, 0
        acc += n
    if start < len(shapes):
        yield start, len(shapes)


def _extract_many(xs, thresholds, duals, flags, to_host) -> list:
    out = []
    for a, b in _chunks([tuple(x.shape) for x in xs]):
        out.extend(extract_batch(xs[a:b], thresholds[a:b], duals[a:b], flags, to_host=to_host))
    return out


def extract_dmsc(scalar_field, persistence_threshold, return_gradient=False, is_dual=False, trace_max_arcs=False,
                 trace_min_arcs=False, trace_max_groups=False, trace_min_groups=False):
    """Mirror of the reference native entry ``dmsc_gpu.extract_dmsc``
    (dmsc/csrc/dmsc_gpu.cpp:128-180, 249-253): 19-tuple for 2-D input, a list
    of 19-tuples for a 3-D batch (computed as device batches, each image's
    outputs identical to a call on it alone)."""
    if scalar_field.dim() not in (2, 3) or scalar_field.dtype != torch.float32 or scalar_field.numel() == 0:
        raise RuntimeError("Input tensor must be a non-empty float32 2D [H, W] or 3D [B, H, W] tensor")
    H, W = int(scalar_field.shape[-2]), int(scalar_field.shape[-1])
    if H + 1 > (2**31 - 1) // 4 // (W + 1):  # input_validation.hxx:24-26
        raise RuntimeError(f"Input is too large for 32-bit cell IDs: {H}x{W}")
    if not torch.cuda.is_available():
        raise RuntimeError("dmsc_b200 requires a CUDA device; there is no CPU compute path")
    on_cpu = scalar_field.device.type != "cuda"
    flags = _flags(return_gradient, is_dual, trace_max_arcs, trace_min_arcs, trace_max_groups, trace_min_groups)
    host_src = None
    if on_cpu:
        xh = scalar_field.contiguous()
        if xh.dim() == 2 and xh.is_pinned():
            # the library uploads the pinned image in bands of rows, each
            # band's gradient starting as soon as its rows have arrived
            host_src = xh
            x = torch.empty(xh.shape, dtype=torch.float32, device="cuda")
        else:
            x = xh.to("cuda", non_blocking=True)
    else:
        x = scalar_field.contiguous()
    with torch.cuda.device(x.device):
        if x.dim() == 2:
            res = extract_single(x, persistence_threshold, flags, host_fixed=on_cpu, host_src=host_src)
            return _to_host(res) if on_cpu else res
        n = x.shape[0]
        return _extract_many(list(x.unbind(0)), [persistence_threshold] * n, [is_dual] * n, flags, on_cpu)


def compute_dmsc_batched(images, persistence_thresholds, is_dual=False, return_gradient=True, trace_valleys=True,
                         trace_ridges=True, trace_peaks=True, trace_basins=True, verbose=False) -> list:
    """Many images of uneven sizes, each with its own threshold and orientation.

    ``images`` is a sequence of 2-D float32 tensors (all CUDA on one device, or
    all CPU); ``persistence_thresholds`` and ``is_dual`` are scalars or one
    value per image. Returns one ``MSComplex`` per image, equal field by field
    to ``compute_dmsc(images[b], persistence_thresholds[b], is_dual=is_dual[b],
    ...)``, computed as device batches (one pass of every stage over the
    union of a batch's images). The reference has no counterpart beyond its
    loop over a 3-D batch of one size and threshold (dmsc/dmsc.py:230-276,
    dmsc/csrc/dmsc_gpu.cpp:84-126).
    """
    images = list(images)
    if not images:
        return []
    n = len(images)
    for x in images:
        if x.dim() != 2:
            raise ValueError(f"Each image must be 2D [H, W]. Got {x.dim()}D.")
        _validate(x)
    thr = list(persistence_thresholds) if hasattr(persistence_thresholds, "__len__") else [persistence_thresholds] * n
    duals = list(is_dual) if hasattr(is_dual, "__len__") else [is_dual] * n
    if len(thr) != n or len(duals) != n:
        raise ValueError("persistence_thresholds and is_dual need one value per image")
    for x in images:
        H, W = int(x.shape[0]), int(x.shape[1])
        if H + 1 > (2**31 - 1) // 4 // (W + 1):
            raise RuntimeError(f"Input is too large for 32-bit cell IDs: {H}x{W}")
    if not torch.cuda.is_available():
        raise RuntimeError("dmsc_b200 requires a CUDA device; there is no CPU compute path")
    devs = {x.device for x in images}
    if len(devs) != 1:
        raise ValueError(f"All images must be on one device. Got {sorted(str(d) for d in devs)}.")
    on_cpu = images[0].device.type != "cuda"
    start = time.perf_counter()
    if on_cpu:
        flat = torch.cat([x.contiguous().reshape(-1) for x in images]).pin_memory().to("cuda", non_blocking=True)
        xs = list(torch.split(flat, [x.numel() for x in images]))
        xs = [v.view(x.shape) for v, x in zip(xs, images)]
    else:
        xs = [x.contiguous() for x in images]
    flags = _flags(return_gradient, False, trace_ridges, trace_valleys, trace_peaks, trace_basins)
    with torch.cuda.device(xs[0].device):
        outs = _extract_many(xs, thr, duals, flags, on_cpu)
    if verbose:
        print(f"Time for MS-complex computation ({n} images): {(time.perf_counter() - start) * 1000:.3f} ms")
    return [MSComplex(*r) for r in outs]


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
