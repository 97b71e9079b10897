"""Batched extraction of images of uneven sizes with per-image thresholds and
orientations (``compute_dmsc_batched`` / ``dmsc_b200_extract_batch``): every
image's outputs equal, bit for bit, the oracle on that image alone."""

import numpy as np
import pytest
import torch

from tests.helpers import diff_fields

pytestmark = pytest.mark.gpu


def _field(rng, kind, H, W):
    if kind == 0:
        a = rng.standard_normal((H, W))
    elif kind == 1:
        a = rng.integers(0, 3, (H, W))
    elif kind == 2:
        a = rng.integers(0, 64, (H, W)) / 64.0
    else:
        y, x = np.mgrid[0:H, 0:W]
        a = np.sin(x / 5.0) * np.cos(y / 7.0) + 0.05 * rng.standard_normal((H, W))
    return torch.from_numpy(a.astype(np.float32))


def _batch(seed, n, lo, hi):
    rng = np.random.default_rng(seed)
    imgs, thr, dual = [], [], []
    for i in range(n):
        H, W = int(rng.integers(lo, hi)), int(rng.integers(lo, hi))
        imgs.append(_field(rng, i % 4, H, W))
        thr.append(float(rng.choice([-1.0, 0.0, 0.05, 0.1, 0.5])))
        dual.append(bool(rng.integers(0, 2)))
    return imgs, thr, dual


def _check(oracle_mod, imgs, thr, dual, got, fl):
    for b, (img, t, d) in enumerate(zip(imgs, thr, dual)):
        exp = oracle_mod.run(img, t, fl[0], d, fl[1], fl[2], fl[3], fl[4])
        assert diff_fields(tuple(got[b]), exp) == [], (b, tuple(img.shape), t, d, fl)


def test_uneven_small_all_outputs(oracle_mod):
    from dmsc_b200 import compute_dmsc_batched

    imgs, thr, dual = _batch(21, 60, 1, 40)
    imgs += [torch.zeros(1, 1), torch.ones(1, 7), torch.arange(5.0).reshape(5, 1)]
    thr += [0.0, 0.1, 0.0]
    dual += [True, False, True]
    got = compute_dmsc_batched([x.cuda() for x in imgs], thr, dual)
    _check(oracle_mod, imgs, thr, dual, got, [True] * 5)


@pytest.mark.parametrize("mask", [0b00000, 0b10101, 0b01010, 0b00110, 0b11001, 0b00010, 0b00100])
def test_uneven_flag_subsets(oracle_mod, mask):
    from dmsc_b200 import compute_dmsc_batched

    fl = [bool(mask >> k & 1) for k in range(5)]  # gradient, ridges, valleys, peaks, basins
    imgs, thr, dual = _batch(100 + mask, 24, 1, 48)
    got = compute_dmsc_batched([x.cuda() for x in imgs], thr, dual, return_gradient=fl[0], trace_ridges=fl[1],
                               trace_valleys=fl[2], trace_peaks=fl[3], trace_basins=fl[4])
    _check(oracle_mod, imgs, thr, dual, got, fl)


def test_uneven_medium_bumps(oracle_mod):
    from dmsc_b200 import compute_dmsc_batched
    from dmsc_b200.synthetic import batch_uneven

    imgs, thr, dual = batch_uneven(12, seed=4, lo=64, hi=384)
    got = compute_dmsc_batched([x.cuda() for x in imgs], thr, dual)
    _check(oracle_mod, imgs, thr, dual, got, [True] * 5)


def test_batched_equals_plain_calls():
    """Batched and plain per-image calls agree on every field (and the batched
    3-D path of compute_dmsc equals per-image calls)."""
    from dmsc_b200 import compute_dmsc, compute_dmsc_batched
    from dmsc_b200.synthetic import batch_uneven

    imgs, thr, dual = batch_uneven(40, seed=9, lo=32, hi=256)
    xs = [x.cuda() for x in imgs]
    got = compute_dmsc_batched(xs, thr, dual)
    for b in range(len(xs)):
        ref = compute_dmsc(xs[b], thr[b], is_dual=dual[b])
        assert diff_fields(tuple(got[b]), tuple(ref)) == [], b
    cube = torch.stack([xs[0][:30, :30], xs[1][:30, :30], xs[2][:30, :30]])
    many = compute_dmsc(cube, 0.05, is_dual=True)
    for b in range(3):
        ref = compute_dmsc(cube[b].clone(), 0.05, is_dual=True)
        assert diff_fields(tuple(many[b]), tuple(ref)) == [], b


def test_cpu_inputs_return_cpu(oracle_mod):
    from dmsc_b200 import compute_dmsc_batched

    imgs, thr, dual = _batch(5, 10, 2, 30)
    got = compute_dmsc_batched(imgs, thr, dual)
    for ms in got:
        assert all(t.device.type == "cpu" for t in ms)
    _check(oracle_mod, imgs, thr, dual, got, [True] * 5)


def test_chunked_batches(oracle_mod, monkeypatch):
    """Batches split into several device batches give the same outputs."""
    from dmsc_b200 import compute_dmsc_batched
    from dmsc_b200 import dmsc as dm

    imgs, thr, dual = _batch(8, 20, 8, 64)
    monkeypatch.setattr(dm, "BATCH_INDEX_CAP", 3000)
    got = compute_dmsc_batched([x.cuda() for x in imgs], thr, dual)
    _check(oracle_mod, imgs, thr, dual, got, [True] * 5)


def test_batch_argument_errors():
    from dmsc_b200 import compute_dmsc_batched

    x = torch.zeros(4, 4, device="cuda")
    with pytest.raises(ValueError):
        compute_dmsc_batched([x, x], [0.1], False)
    with pytest.raises(ValueError):
        compute_dmsc_batched([torch.zeros(2, 3, 3, device="cuda")], 0.1)
    with pytest.raises(TypeError):
        compute_dmsc_batched([x.double()], 0.1)
    assert compute_dmsc_batched([], 0.1) == []


def test_sharded_single_rank_matches_plain_calls():
    """The sharded driver on one rank (no process group) equals plain calls."""
    from dmsc_b200 import compute_dmsc
    from dmsc_b200.sharding import compute_dmsc_sharded

    imgs, thr, dual = _batch(31, 12, 2, 64)
    full = compute_dmsc_sharded(imgs, thr, dual, device="cuda:0", gather=True)
    for b, ms in enumerate(full):
        ref = compute_dmsc(imgs[b], thr[b], is_dual=dual[b])
        assert diff_fields(tuple(ms), tuple(ref)) == [], b
