"""Differentiable persistence values.

Every persistence value the complex reports (``p_min``, ``p_max``) is the
float32 difference of two input pixels: the value pixel of a saddle and the
value pixel of the extremum that dies at it (dmsc/csrc/cpu/persistence.hxx:
82-104, 139-161; a cell's value pixel is its highest vertex in the primal,
its lowest in the dual, dmsc/csrc/cpu/cell_compare.hxx:33-87). On a field
without ties the pairing does not change under a small enough perturbation,
so d p / d img is +1 on one pixel and -1 on the other, and the gradient of
any loss of the persistence values scatters dL/dp onto those pixel pairs.

``persistence_pairs`` runs the pairing on the GPU (no gradient field, arcs or
labels are built) and returns the values with their pixel pairs; its
backward is one deterministic device scatter (``dmsc_b200_scatter_pair_grads``:
stable sort by pixel and a segmented sum in a fixed order, no float
atomics), so repeated backward passes give identical bits. The reference has
no counterpart: its outputs carry no gradient.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _lib
from .dmsc import _batch_raw, _ptr, _validate


@dataclass
class PersistencePairs:
    """Persistence pairs of a field or a batch, min side then max side.

    ``persistence``: float32 [n], differentiable with respect to the input;
    per image the entries of ``p_min`` followed by ``p_max`` (bit-identical to
    those outputs of ``compute_dmsc`` with the same threshold), images in
    order. ``image``: int64 [n] image index. ``side``: int8 [n], 0 for a
    ``p_min`` entry, 1 for ``p_max``. ``ppairs``: int32 [n], the matching
    ``ppairs_min`` / ``ppairs_max`` entry (-1 for a cycle). ``plus_pixel`` /
    ``minus_pixel``: int32 [n] image-local pixel ids (y * W + x) with
    ``persistence = img[plus] - img[minus]``; -1 for a cycle, whose
    persistence is the constant -1.
    """

    persistence: torch.Tensor
    image: torch.Tensor
    side: torch.Tensor
    ppairs: torch.Tensor
    plus_pixel: torch.Tensor
    minus_pixel: torch.Tensor


def _run(x3, thresholds, duals):
    """Forward on a contiguous [B, H, W] CUDA tensor: the values, metadata and
    the pixel pairs as flat pixel ids of ``x3`` (-1 for cycles)."""
    B, H, W = x3.shape
    imgs = list(x3.unbind(0))
    out, lens, _, _, _, _ = _batch_raw(imgs, thresholds, duals, 0, flat=x3.reshape(-1), pair_pixels=True)
    dev = x3.device
    n_min = torch.tensor(lens["p_min"], device=dev)
    n_max = torch.tensor(lens["p_max"], device=dev)
    ids = torch.arange(B, device=dev)
    img_min = torch.repeat_interleave(ids, n_min)
    img_max = torch.repeat_interleave(ids, n_max)
    # per image: its p_min entries, then its p_max entries
    order_key = torch.cat([img_min * 2, img_max * 2 + 1])
    perm = torch.sort(order_key, stable=True).indices
    cat = lambda a, b: torch.cat([a, b])[perm]  # noqa: E731
    p = cat(out["p_min"], out["p_max"])
    image = cat(img_min, img_max)
    side = cat(torch.zeros_like(img_min, dtype=torch.int8), torch.ones_like(img_max, dtype=torch.int8))
    ppairs = cat(out["ppairs_min"], out["ppairs_max"])
    plus = cat(out["plus_min"], out["plus_max"])
    minus = cat(out["minus_min"], out["minus_max"])
    base = (image * (H * W)).to(torch.int32)
    plus_g = torch.where(plus >= 0, plus + base, plus)
    minus_g = torch.where(minus >= 0, minus + base, minus)
    return p, image, side, ppairs, plus, minus, plus_g, minus_g


class _PersistenceFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x3, thresholds, duals):
        p, image, side, ppairs, plus, minus, plus_g, minus_g = _run(x3, thresholds, duals)
        ctx.save_for_backward(plus_g, minus_g)
        ctx.shape = x3.shape
        ctx.mark_non_differentiable(image, side, ppairs, plus, minus)
        return p, image, side, ppairs, plus, minus

    @staticmethod
    def backward(ctx, grad_p, *unused):
        plus_g, minus_g = ctx.saved_tensors
        return scatter_pair_grads(plus_g, minus_g, grad_p, ctx.shape), None, None


def scatter_pair_grads(plus, minus, grad, shape):
    """grad_img (float32, ``shape``) = sum over i of +grad[i] at flat pixel
    ``plus[i]`` and -grad[i] at ``minus[i]`` (ends of -1 skipped), summed in a
    fixed order on the device (deterministic, no float atomics)."""
    dev = plus.device
    out = torch.empty(shape, dtype=torch.float32, device=dev)
    plus = plus.to(torch.int32).contiguous()
    minus = minus.to(torch.int32).contiguous()
    g = grad.to(torch.float32).contiguous() if grad is not None else torch.zeros(plus.numel(), device=dev)
    ctx = _lib.context(dev.index if dev.index is not None else torch.cuda.current_device())
    st = torch.cuda.current_stream(dev)
    ctx.check(ctx.lib.dmsc_b200_scatter_pair_grads(ctx.h, _ptr(plus), _ptr(minus), _ptr(g), plus.numel(), _ptr(out),
                                                   out.numel(), ctypes.c_void_p(st.cuda_stream)),
              "dmsc_b200_scatter_pair_grads")
    return out


def persistence_pairs(img, persistence_threshold, is_dual=False) -> PersistencePairs:
    """Differentiable persistence values of a 2-D [H, W] field or a 3-D
    [B, H, W] batch (float32, CUDA). ``persistence_threshold`` and ``is_dual``
    are scalars or one value per image, with the meaning they have in
    ``compute_dmsc``: pairs with persistence <= threshold are cancelled and do
    not appear (a negative threshold keeps every pair). Gradients flow to
    ``img`` through ``persistence`` only; they are exact where the field has
    no ties."""
    _validate(img)
    if img.device.type != "cuda":
        raise RuntimeError("persistence_pairs needs a CUDA tensor; there is no CPU compute path")
    x3 = (img.unsqueeze(0) if img.dim() == 2 else img).contiguous()
    B = x3.shape[0]
    thr = list(persistence_threshold) if hasattr(persistence_threshold, "__len__") else [persistence_threshold] * B
    duals = list(is_dual) if hasattr(is_dual, "__len__") else [is_dual] * B
    if len(thr) != B or len(duals) != B:
        raise ValueError("persistence_threshold and is_dual need one value per image")
    H, W = int(x3.shape[1]), int(x3.shape[2])
    if H + 1 > (2**31 - 1) // 4 // (W + 1):
        raise RuntimeError(f"Input is too large for 32-bit cell IDs: {H}x{W}")
    with torch.cuda.device(x3.device):
        p, image, side, ppairs, plus, minus = _PersistenceFn.apply(x3, [float(t) for t in thr],
                                                                   [bool(d) for d in duals])
    return PersistencePairs(p, image, side, ppairs, plus, minus)


def topological_loss(img, persistence_threshold=-1.0, max_persistence=0.1, is_dual=False):
    """Topological denoising loss: sum of p^2 over the pairs with
    ``ppairs != -1`` and ``0 <= p < max_persistence``."""
    pp = persistence_pairs(img, persistence_threshold, is_dual)
    p = pp.persistence
    keep = (pp.ppairs != -1) & (p >= 0) & (p < max_persistence)
    return (p * p * keep).sum()
