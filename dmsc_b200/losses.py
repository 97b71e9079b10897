"""Topological loss functions on top of the differentiable persistence pairs.

The reference lists loss functions for topological segmentation as future
work (readme.md, TODOs); it has no counterpart. Every loss here is a plain
torch function of the persistence values returned by
``autograd.persistence_pairs``, so its gradient reaches the image through the
deterministic pixel-pair scatter (no float atomics), and per-image sums are
segmented reductions in a fixed order: repeated forward and backward passes
give identical bits. Each loss has a ``*_from_pairs`` form that takes the
values and their metadata directly (any float dtype), which is also how the
tests evaluate the same loss in FP64 for finite differences.

Conventions (public sides, as in ``compute_dmsc``): side 0 is the min side
(``p_min``: minima, whose regions are the basins), side 1 the max side
(``p_max``: maxima, the peaks). A cycle (``ppairs == -1``, persistence -1)
is never part of a loss. Each image keeps one essential extremum per side
that never dies, so an image with ``k`` regions on a side has ``k - 1``
finite pairs above the simplification threshold.
"""

from __future__ import annotations

import torch

from .autograd import persistence_pairs

_SIDES = {"min": (0,), "max": (1,), "both": (0, 1)}


def _per_image_sum(term, image, B):
    """Per-image sums in a fixed order (segmented reduction over the entries
    grouped by image): deterministic bits, unlike a float index_add."""
    if term.numel() == 0:
        return torch.zeros(B, dtype=term.dtype, device=term.device)
    order = torch.sort(image, stable=True).indices
    lengths = torch.bincount(image, minlength=B)
    return torch.segment_reduce(term[order], "sum", lengths=lengths, unsafe=True)


def _side_mask(side_t, ppairs, p, side):
    if side not in _SIDES:
        raise ValueError(f"side must be one of {sorted(_SIDES)}, got {side!r}")
    m = torch.zeros_like(ppairs, dtype=torch.bool)
    for s in _SIDES[side]:
        m |= side_t == s
    return m & (ppairs != -1) & (p >= 0)


def denoising_loss_from_pairs(p, image, side_t, ppairs, max_persistence=0.1, side="both", n_images=None):
    """Per image: sum of p^2 over the finite pairs of ``side`` with
    ``0 <= p < max_persistence`` (noise-level features pushed to zero
    persistence). Returns a [B] tensor."""
    B = int(n_images if n_images is not None else (int(image.max()) + 1 if image.numel() else 0))
    keep = _side_mask(side_t, ppairs, p, side) & (p < max_persistence)
    return _per_image_sum(torch.where(keep, p * p, torch.zeros_like(p)), image, B)


def _ranks_desc(p, image, mask):
    """Rank of every entry among the masked entries of its image by
    descending persistence (ties by position: deterministic); -1 if not
    masked."""
    n = p.numel()
    idx = torch.arange(n, device=p.device)
    key_p = torch.where(mask, p.detach(), torch.full_like(p.detach(), -float("inf")))
    o1 = torch.sort(key_p, descending=True, stable=True).indices
    o2 = torch.sort(image[o1], stable=True).indices
    order = o1[o2]  # by image, then descending p
    img_sorted = image[order]
    start = torch.searchsorted(img_sorted, img_sorted, right=False)
    rank = torch.empty(n, dtype=torch.int64, device=p.device)
    rank[order] = idx - start
    return torch.where(mask, rank, torch.full_like(rank, -1))


def betti_loss_from_pairs(p, image, side_t, ppairs, n_regions, side="min", target=1.0, n_images=None):
    """Betti-number prior (Clough et al., "A topological loss function for
    deep-learning based image segmentation using persistent homology"): per
    image, the ``n_regions - 1`` most persistent finite pairs of ``side`` are
    pulled to persistence ``target`` and every other one to 0:
    sum_{rank < k-1} (target - p)^2 + sum_{rank >= k-1} p^2. ``n_regions``
    is an int or one int per image. Returns a [B] tensor."""
    B = int(n_images if n_images is not None else (int(image.max()) + 1 if image.numel() else 0))
    mask = _side_mask(side_t, ppairs, p, side)
    k = torch.as_tensor(n_regions, dtype=torch.int64, device=p.device).reshape(-1)
    if k.numel() == 1:
        k = k.expand(B)
    if k.numel() != B:
        raise ValueError("n_regions needs one value per image")
    if bool((k < 1).any()):
        raise ValueError("n_regions must be >= 1 (the essential region)")
    rank = _ranks_desc(p, image, mask)
    top = mask & (rank < (k[image] - 1))
    term = torch.where(top, (target - p) ** 2, p * p)
    term = torch.where(mask, term, torch.zeros_like(p))
    return _per_image_sum(term, image, B)


def _pairs(img, persistence_threshold, is_dual):
    pp = persistence_pairs(img, persistence_threshold, is_dual)
    B = 1 if img.dim() == 2 else int(img.shape[0])
    return pp, B


def denoising_loss(img, max_persistence=0.1, side="both", persistence_threshold=-1.0, is_dual=False,
                   reduction="sum"):
    """Topological denoising of one side or both: the sum of p^2 over pairs
    with 0 <= p < ``max_persistence`` (``side="both"`` is the loss of
    ``autograd.topological_loss``)."""
    pp, B = _pairs(img, persistence_threshold, is_dual)
    per = denoising_loss_from_pairs(pp.persistence, pp.image, pp.side, pp.ppairs, max_persistence, side, B)
    return _reduce(per, reduction)


def betti_loss(img, n_regions, side="min", target=1.0, persistence_threshold=-1.0, is_dual=False, reduction="sum"):
    """Betti-number prior on one side: ``n_regions`` basins (``side="min"``)
    or peaks (``side="max"``) per image; see betti_loss_from_pairs."""
    pp, B = _pairs(img, persistence_threshold, is_dual)
    per = betti_loss_from_pairs(pp.persistence, pp.image, pp.side, pp.ppairs, n_regions, side, target, B)
    return _reduce(per, reduction)


def segmentation_loss(img, n_basins=None, n_peaks=None, target=1.0, persistence_threshold=-1.0, is_dual=False,
                      reduction="sum"):
    """Topological segmentation prior: the Betti loss of the basins (min
    side) with ``n_basins`` regions plus that of the peaks (max side) with
    ``n_peaks`` regions, from one forward of the pairing. A side given as
    None is left free."""
    if n_basins is None and n_peaks is None:
        raise ValueError("give n_basins, n_peaks or both")
    pp, B = _pairs(img, persistence_threshold, is_dual)
    per = torch.zeros(B, dtype=pp.persistence.dtype, device=pp.persistence.device)
    if n_basins is not None:
        per = per + betti_loss_from_pairs(pp.persistence, pp.image, pp.side, pp.ppairs, n_basins, "min", target, B)
    if n_peaks is not None:
        per = per + betti_loss_from_pairs(pp.persistence, pp.image, pp.side, pp.ppairs, n_peaks, "max", target, B)
    return _reduce(per, reduction)


def _reduce(per, reduction):
    if reduction == "sum":
        return per.sum()
    if reduction == "mean":
        return per.mean()
    if reduction == "none":
        return per
    raise ValueError(f"reduction must be 'sum', 'mean' or 'none', got {reduction!r}")
