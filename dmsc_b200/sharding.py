"""Image-level sharding of a batch over the GPUs of one node.

Images are independent units of ``compute_dmsc``: nothing crosses between
them, so a batch shards across ranks with no data-path collective. One image
is never split across GPUs: its persistence pairing and arc simplification
are global union-find problems over the whole image (the reference runs them
sequentially per image, dmsc/csrc/cpu/persistence.hxx:16-182,
dmsc/csrc/cpu/arcs_simplification.hxx:310-504), so within an image the only
multi-GPU form is replicas.

One process per GPU (``torchrun``); every rank holds the same list of images
(or just their shapes) and computes the same plan on its own, so the plan
needs no exchange. Each rank computes its shard as device batches on its own
GPU (``compute_dmsc_batched``); results stay on the rank unless ``gather``
asks for every image on every rank (one ``all_gather_object`` of CPU
results, the only collective here).
"""

from __future__ import annotations

import heapq


def shard_plan(shapes, world: int) -> list:
    """Partition of image indices over ``world`` ranks balanced by pixel count.

    Longest-processing-time greedy: images by descending area (ties by
    index) go to the rank with the least assigned area (ties by rank). Each
    rank's list is returned in ascending image order. Deterministic, so every
    rank derives the same plan from the same shapes.
    """
    if world < 1:
        raise ValueError(f"world must be >= 1. Got {world}.")
    areas = [int(h) * int(w) for h, w in shapes]
    order = sorted(range(len(areas)), key=lambda i: (-areas[i], i))
    heap = [(0, r) for r in range(world)]
    plan = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        plan[r].append(i)
        heapq.heappush(heap, (load + areas[i], r))
    return [sorted(p) for p in plan]


def local_shard(shapes, world: int, rank: int) -> list:
    """Image indices of ``rank`` in the plan of :func:`shard_plan`."""
    if not 0 <= rank < world:
        raise ValueError(f"rank must be in [0, {world}). Got {rank}.")
    return shard_plan(shapes, world)[rank]


def _default_compute(images, thresholds, duals, device, **kwargs):
    import torch

    from .dmsc import compute_dmsc_batched

    xs = [x.to(device, non_blocking=True) for x in images]
    with torch.cuda.device(device):
        return compute_dmsc_batched(xs, thresholds, duals, **kwargs)


def compute_dmsc_sharded(images, persistence_thresholds, is_dual=False, group=None, device=None, gather=False,
                         compute=None, **kwargs):
    """Computes this rank's share of a batch of uneven images.

    ``images`` is the whole batch (the same sequence on every rank);
    ``persistence_thresholds`` and ``is_dual`` are scalars or one value per
    image. The rank and world come from ``torch.distributed`` (``group``) when
    it is initialised, else a single rank. ``device`` defaults to
    ``cuda:<LOCAL_RANK>``. ``kwargs`` go to ``compute_dmsc_batched``
    (``return_gradient``, ``trace_*``).

    Returns ``{image index: MSComplex}`` for this rank's images; with
    ``gather`` every rank receives the list of all images' results (on the
    CPU) in image order. ``compute`` replaces the device computation with
    ``compute(images, thresholds, duals, device, **kwargs) -> list`` (for
    host-side tests).
    """
    import os

    import torch.distributed as dist

    images = list(images)
    n = len(images)
    thr = list(persistence_thresholds) if hasattr(persistence_thresholds, "__len__") else [persistence_thresholds] * n
    duals = list(is_dual) if hasattr(is_dual, "__len__") else [is_dual] * n
    if len(thr) != n or len(duals) != n:
        raise ValueError("persistence_thresholds and is_dual need one value per image")
    if dist.is_available() and dist.is_initialized():
        world, rank = dist.get_world_size(group), dist.get_rank(group)
    else:
        world, rank = 1, 0
    if device is None:
        device = f"cuda:{int(os.environ.get('LOCAL_RANK', '0'))}"
    mine = local_shard([tuple(x.shape[-2:]) for x in images], world, rank)
    fn = compute if compute is not None else _default_compute
    res = fn([images[i] for i in mine], [thr[i] for i in mine], [duals[i] for i in mine], device, **kwargs) if mine \
        else []
    local = dict(zip(mine, res))
    if not gather:
        return local
    if world == 1:
        return [_to_cpu(local[i]) for i in range(n)]
    parts = [None] * world
    dist.all_gather_object(parts, {i: _to_cpu(v) for i, v in local.items()}, group=group)
    merged = {}
    for p in parts:
        merged.update(p)
    return [merged[i] for i in range(n)]


def _to_cpu(ms):
    """An MSComplex (or a tensor, or a plain value) with its tensors on the CPU."""
    from dataclasses import fields, is_dataclass, replace

    if is_dataclass(ms):
        return replace(ms, **{f.name: getattr(ms, f.name).cpu() for f in fields(ms)
                              if hasattr(getattr(ms, f.name), "cpu")})
    return ms.cpu() if hasattr(ms, "cpu") else ms
