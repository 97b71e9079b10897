"""The C oracle against the reference: its golden fixtures, the reference's own
fixtures and (when built) the compiled reference on random fields. CPU only."""

import os
import sys

import numpy as np
import pytest
import torch

from tests.helpers import FIELDS, diff_fields, golden_cases, load_golden

REF_DATA = "/root/reference/tests/data"
REF_LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


@pytest.mark.parametrize("name,path", list(golden_cases()))
def test_oracle_matches_golden(oracle_mod, name, path):
    img, thr, dual, fl, expected = load_golden(path)
    got = oracle_mod.run(img, thr, fl[0], dual, fl[1], fl[2], fl[3], fl[4])
    assert diff_fields(got, expected) == []


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference fixtures not present")
@pytest.mark.parametrize("dual", [False, True])
@pytest.mark.parametrize("flt,thr", [("raw", -1.0), ("flt", 0.15)])
def test_oracle_matches_reference_fixtures(oracle_mod, dual, flt, thr):
    """The reference's own single-thread fixtures (tests/data/ms_st_*.pt),
    compared field by field and exactly."""
    img = torch.load(os.path.join(REF_DATA, "landscape_32x32.pt"))
    gt = torch.load(os.path.join(REF_DATA, f"ms_st_{'dual' if dual else 'primal'}_{flt}.pt"), weights_only=False)
    got = dict(zip(FIELDS, oracle_mod.run(img, thr, True, dual, True, True, True, True)))
    for k, v in gt.items():
        if v is None:
            continue
        assert torch.equal(v, got[k]), k


def _ref():
    if not os.path.exists(os.path.join(REF_LIB, "dmsc_cpu.so")):
        return None
    sys.path.insert(0, REF_LIB)
    import dmsc_cpu

    return dmsc_cpu


@pytest.mark.skipif(_ref() is None, reason="reference checker not built (oracle/build_ref.py)")
def test_oracle_matches_reference_random(oracle_mod):
    ref = _ref()
    torch.set_num_threads(1)
    rng = np.random.default_rng(42)
    for it in range(150):
        H, W = int(rng.integers(1, 26)), int(rng.integers(1, 26))
        kind = it % 4
        if kind == 0:
            a = rng.standard_normal((H, W))
        elif kind == 1:
            a = rng.integers(0, 3, (H, W))
        elif kind == 2:
            a = rng.integers(0, 64, (H, W)) / 64.0
        else:
            a = np.sin(np.arange(W)[None, :] / 3.0) * np.cos(np.arange(H)[:, None] / 4.0) + 0.05 * rng.standard_normal((H, W))
        img = torch.from_numpy(a.astype(np.float32))
        thr = float(rng.choice([-1.0, 0.0, 0.1, 0.5, 2.0]))
        dual = bool(rng.integers(0, 2))
        fl = [bool(v) for v in rng.integers(0, 2, 5)]
        r = ref.extract_dmsc(img, thr, fl[0], dual, fl[1], fl[2], fl[3], fl[4])
        exp = [r[i] for i in range(19)]
        got = oracle_mod.run(img, thr, fl[0], dual, fl[1], fl[2], fl[3], fl[4])
        assert diff_fields(got, exp) == [], (it, H, W, thr, dual, fl)
