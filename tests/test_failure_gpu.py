"""Failure handling of the device loops and host waits (no GPU fault is made).

Every loop of the pipeline has a bound no input reaches; a test-only setter
lowers the pairing-round, replay-round and expansion-level bounds so each one
runs out on a small field. The call must raise RuntimeError with the
iteration-cap message, and the next normal call on the same context must be
bit-exact again. A host wait deadline shorter than the work must end the call
with an error instead of spinning.
"""

import pytest
import torch

from tests.helpers import diff_fields

pytestmark = pytest.mark.gpu


def _field():
    from dmsc_b200.synthetic import field_256_bumps

    return field_256_bumps(seed=31).cuda()


def _run(img, thr=0.1):
    from dmsc_b200 import extract_dmsc

    return extract_dmsc(img, thr, True, False, True, True, True, True)


@pytest.mark.parametrize("which", ["pair_rounds", "replay_rounds", "emit_levels"])
def test_loop_cap_raises_and_context_recovers(which):
    from dmsc_b200 import _lib

    img = _field()
    ref = _run(img)
    ctx = _lib.context(torch.cuda.current_device())
    counts = ctx.loop_counts()
    needed = {"pair_rounds": counts["pair_rounds_faces"], "replay_rounds": counts["replay_rounds_faces"],
              "emit_levels": counts["emit_levels_faces"]}[which]
    assert needed > 1, counts  # the cap of 1 must cut the loop short
    try:
        ctx.set_loop_caps(**{which: 1})
        with pytest.raises(RuntimeError, match="bounded device loop reached its cap"):
            _run(img)
    finally:
        ctx.set_loop_caps()
    assert diff_fields(_run(img), ref) == []


def test_wait_deadline_raises():
    """A private context with a wait deadline far below the work's duration:
    the first readback gives up with an error. The context is destroyed
    afterwards (the work may still be running), as the header asks."""
    import ctypes

    from dmsc_b200 import _lib
    from dmsc_b200.synthetic import field_4096_bumps

    img = field_4096_bumps(seed=7).cuda()
    torch.cuda.synchronize()
    ctx = _lib.Context(torch.cuda.current_device())
    try:
        ctx.set_wait_timeout(1e-9)
        H, W = img.shape
        sz = _lib.Sizes()
        peaks = torch.empty((H + 1, W + 1), dtype=torch.int32, device="cuda")
        basins = torch.empty((H, W), dtype=torch.int32, device="cuda")
        rc = ctx.lib.dmsc_b200_extract(ctx.h, ctypes.c_void_p(img.data_ptr()), H, W, ctypes.c_float(0.05),
                                       _lib.TRACE_PEAKS | _lib.TRACE_BASINS, None, ctypes.c_void_p(peaks.data_ptr()),
                                       ctypes.c_void_p(basins.data_ptr()), ctypes.byref(sz),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 3  # DMSC_B200_ERR_CUDA
        assert "did not finish within" in ctx.lib.dmsc_b200_last_error(ctx.h).decode()
    finally:
        ctx.close()
        torch.cuda.synchronize()
    # other contexts are unaffected
    ref = _run(_field())
    assert diff_fields(_run(_field()), ref) == []
