"""Launch shapes change speed only: every gradient tile shape, label tile
shape, pairing, replay and expansion batch shape and persistent-kernel
residency gives the same
bits; the tuner runs,
reports and caches a choice that later calls of the size class use."""

import itertools

import pytest
import torch

from tests.helpers import diff_fields

pytestmark = pytest.mark.gpu


def test_every_launch_shape_is_bit_identical():
    from dmsc_b200 import _lib, extract_dmsc, tuning
    from dmsc_b200.synthetic import field_4096_bumps

    img = field_4096_bumps(seed=77, size=700).cuda()
    tuning.clear()
    ctx = _lib.context(torch.cuda.current_device())
    lim = ctx.tuning_limits()
    ref = {d: extract_dmsc(img, 0.05, True, d, True, True, True, True) for d in (False, True)}
    tuning._tuning.active = True  # keep the shapes set below for the calls
    try:
        for g, lab, pb, sc, ps in itertools.product(range(lim["grad_shapes"]), range(lim["label_shapes"]), (0, 1, 3),
                                                    range(1, lim["seg_cursors"] + 1), range(lim["pair_shapes"])):
            ctx.set_tuning(grad_shape=g, label_shape=lab, pair_blocks_per_sm=pb, replay_blocks_per_sm=pb,
                           emit_blocks_per_sm=pb, seg_cursors=sc, pair_shape=ps, replay_shape=ps, emit_shape=ps)
            for d in (False, True):
                got = extract_dmsc(img, 0.05, True, d, True, True, True, True)
                assert diff_fields(got, ref[d]) == [], (g, lab, pb, sc, ps, d)
    finally:
        tuning._tuning.active = False
        ctx.set_tuning(**tuning._default_tuning())
        ctx._applied_tuning = None


def test_tune_reports_and_caches():
    from dmsc_b200 import _lib, compute_dmsc, tuning
    from dmsc_b200.synthetic import field_4096_bumps

    img = field_4096_bumps(seed=78, size=512).cuda()
    tuning.clear()
    try:
        rep = tuning.tune(lambda: compute_dmsc(img, 0.05), img.numel(), reps=3)
        assert set(rep["choice"]) == set(tuning._default_tuning())
        assert rep["default_ms"] > 0 and rep["tuned_ms"] > 0
        assert set(rep["stages"]) == {t[0] for t in tuning.TUNABLES}
        assert tuning.choice(torch.cuda.current_device(), img.numel()) == rep["choice"]
        ctx = _lib.context(torch.cuda.current_device())
        compute_dmsc(img, 0.05)
        t = ctx.get_tuning()
        assert {k: getattr(t, k) for k in rep["choice"]} == rep["choice"]
    finally:
        tuning.clear()
