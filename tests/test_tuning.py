"""Selection logic of the launch-shape tuner (dmsc_b200.tuning), on fake
timings and a fake context (CPU)."""

import pytest

from dmsc_b200 import tuning


def test_select_median_and_ties():
    assert tuning.select({0: [5.0, 1.0, 9.0], 1: [4.0, 4.0, 4.0], 2: [6.0]}) == 1  # medians 5, 4, 6
    assert tuning.select({0: [2.0, 2.0], 1: [2.0, 2.0]}) == 0  # a tie keeps the first (the default)
    assert tuning.select({0: [], 3: [1.0]}) == 3
    assert tuning.select({}) is None
    # one outlier does not move the median
    assert tuning.select({0: [1.0, 1.1, 50.0], 1: [1.2, 1.2, 1.2]}) == 0


def test_block_candidates_and_size_class():
    assert tuning._blocks(6) == [0, 1, 2, 4]
    assert tuning._blocks(1) == [0]
    assert tuning._blocks(8) == [0, 1, 2, 4]
    assert tuning.size_class(4096 * 4096) == 24
    assert tuning.size_class(4096 * 4096 - 1) == 23
    assert tuning.size_class(0) == 0


class _FakeCtx:
    def __init__(self, device=0):
        self.device = device
        self.calls = []

    def set_tuning(self, **kw):
        self.calls.append(dict(kw))


def test_apply_uses_cache_per_device_and_class():
    tuning.clear()
    ctx = _FakeCtx()
    tuning.apply(ctx, 1000)  # never tuned: the defaults
    assert ctx.calls == [tuning._default_tuning()]
    tuning.apply(ctx, 1000)  # unchanged: no new call
    assert len(ctx.calls) == 1
    choice = dict(tuning._default_tuning(), grad_shape=2, pair_blocks_per_sm=4)
    with tuning._lock:
        tuning._cache[(0, tuning.size_class(4096 * 4096))] = choice
    tuning.apply(ctx, 4096 * 4096)
    assert ctx.calls[-1] == choice
    tuning.apply(ctx, 1000)
    assert ctx.calls[-1] == tuning._default_tuning()
    other = _FakeCtx(device=1)
    tuning.apply(other, 4096 * 4096)  # another device: its own cache
    assert other.calls == [tuning._default_tuning()]
    tuning._tuning.active = True
    try:
        n = len(ctx.calls)
        tuning.apply(ctx, 4096 * 4096)
        assert len(ctx.calls) == n  # no-op while tuning
    finally:
        tuning._tuning.active = False
    tuning.clear()


@pytest.mark.parametrize("name", [t[0] for t in tuning.TUNABLES])
def test_tunables_name_real_stages(name):
    from dmsc_b200 import _lib

    stage = dict((t[0], t[1]) for t in tuning.TUNABLES)[name]
    assert stage in _lib.STAGES
    assert name in tuning._default_tuning()
