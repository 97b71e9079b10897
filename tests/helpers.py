"""Comparison helpers shared by the tests."""

from __future__ import annotations

import glob
import os

import numpy as np
import torch

FIELDS = (
    "shape max_pts min_pts sad_pts e_max e_min p_max p_min ppairs_max ppairs_min grad_indices "
    "peaks ridges ridge_offsets ridge_arc_offsets basins valleys valley_offsets valley_arc_offsets"
).split()
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def as_np(t):
    if isinstance(t, torch.Tensor):
        return t.detach().cpu().numpy()
    return np.asarray(t)


def diff_fields(actual, expected):
    """Names of the fields that differ bit for bit (float32 compared by bits,
    so -0.0 != +0.0 and NaN payloads must agree)."""
    bad = []
    for name, a, e in zip(FIELDS, actual, expected):
        a, e = as_np(a), as_np(e)
        if a.shape != e.shape or a.dtype != e.dtype:
            bad.append(f"{name}: shape/dtype {a.shape}/{a.dtype} vs {e.shape}/{e.dtype}")
            continue
        if a.dtype == np.float32:
            same = np.array_equal(a.view(np.int32), e.view(np.int32))
        else:
            same = np.array_equal(a, e)
        if not same:
            bad.append(name)
    return bad


def golden_cases():
    for p in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        yield os.path.basename(p)[:-4], p


def load_golden(path):
    z = np.load(path)
    img = torch.from_numpy(z["image"])
    fl = [bool(v) for v in z["flags"]]
    expected = tuple(torch.from_numpy(z[f]) for f in FIELDS)
    return img, float(z["threshold"]), bool(z["is_dual"]), fl, expected
