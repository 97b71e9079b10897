"""Parity of the CUDA path (through the C ABI) with the reference: bit-exact on
every output against the golden fixtures and the C oracle."""

import numpy as np
import pytest
import torch

from tests.helpers import FIELDS, diff_fields, golden_cases, load_golden

pytestmark = pytest.mark.gpu


def gpu_run(img, thr, fl, dual):
    from dmsc_b200 import extract_dmsc

    return extract_dmsc(img.cuda(), thr, fl[0], dual, fl[1], fl[2], fl[3], fl[4])


@pytest.mark.parametrize("name,path", list(golden_cases()))
def test_golden(name, path):
    img, thr, dual, fl, expected = load_golden(path)
    got = gpu_run(img, thr, fl, dual)
    assert diff_fields(got, expected) == []


def _random_field(rng, kind, H, W):
    if kind == 0:
        a = rng.standard_normal((H, W))
    elif kind == 1:
        a = rng.integers(0, 3, (H, W))
    elif kind == 2:
        a = rng.integers(0, 64, (H, W)) / 64.0
    elif kind == 3:
        a = rng.random((H, W))
    else:
        y, x = np.mgrid[0:H, 0:W]
        a = np.sin(x / 5.0) * np.cos(y / 7.0) + 0.05 * rng.standard_normal((H, W))
    return torch.from_numpy(a.astype(np.float32))


def test_random_small_vs_oracle(oracle_mod):
    rng = np.random.default_rng(7)
    for it in range(250):
        H, W = int(rng.integers(1, 40)), int(rng.integers(1, 40))
        img = _random_field(rng, it % 5, H, W)
        thr = float(rng.choice([-1.0, 0.0, 0.05, 0.1, 0.5, 2.0]))
        dual = bool(rng.integers(0, 2))
        fl = [bool(v) for v in rng.integers(0, 2, 5)]
        exp = oracle_mod.run(img, thr, fl[0], dual, fl[1], fl[2], fl[3], fl[4])
        got = gpu_run(img, thr, fl, dual)
        assert diff_fields(got, exp) == [], (it, H, W, thr, dual, fl)


@pytest.mark.parametrize("dual", [False, True])
@pytest.mark.parametrize("thr", [0.0, 0.1])
def test_bump_256(oracle_mod, dual, thr):
    from dmsc_b200.synthetic import field_256_bumps

    img = field_256_bumps(seed=3)
    exp = oracle_mod.run(img, thr, True, dual, True, True, True, True)
    got = gpu_run(img, thr, [True] * 5, dual)
    assert diff_fields(got, exp) == []


@pytest.mark.parametrize("dual", [False, True])
@pytest.mark.parametrize("thr", [0.0, 0.05])
def test_bump_1024(oracle_mod, dual, thr):
    from dmsc_b200.synthetic import field_4096_bumps

    img = field_4096_bumps(seed=5, size=1024)
    exp = oracle_mod.run(img, thr, True, dual, True, True, True, True)
    got = gpu_run(img, thr, [True] * 5, dual)
    assert diff_fields(got, exp) == []


def test_uniform_ties(oracle_mod):
    """i.i.d. 12-bit uniform values: heavy ties and zero-persistence pairs."""
    rng = np.random.default_rng(11)
    for thr, size in ((0.0, 512), (0.5, 96)):
        img = torch.from_numpy((rng.integers(0, 1 << 12, (size, size)) / (1 << 12)).astype(np.float32))
        for dual in (False, True):
            exp = oracle_mod.run(img, thr, True, dual, True, True, True, True)
            got = gpu_run(img, thr, [True] * 5, dual)
            assert diff_fields(got, exp) == [], (thr, size, dual)


def test_batch_matches_sequential():
    from dmsc_b200 import compute_dmsc

    fields = torch.randn((3, 9, 7), generator=torch.Generator().manual_seed(8)).cuda()
    batched = compute_dmsc(fields, 0.15)
    sequential = [compute_dmsc(f, 0.15) for f in fields]
    for a, b in zip(batched, sequential):
        assert diff_fields(list(a), list(b)) == []
        assert all(x.device == y.device for x, y in zip(a, b))


def test_noncontiguous_input():
    from dmsc_b200 import compute_dmsc

    field = torch.randn((7, 11), generator=torch.Generator().manual_seed(4)).cuda().transpose(0, 1)
    assert not field.is_contiguous()
    assert diff_fields(list(compute_dmsc(field, 0.1)), list(compute_dmsc(field.contiguous(), 0.1))) == []


def test_cpu_input_returns_cpu_outputs(oracle_mod):
    from dmsc_b200 import compute_dmsc

    img = torch.randn((13, 10), generator=torch.Generator().manual_seed(2))
    ms = compute_dmsc(img, 0.1)
    assert all(t.device.type == "cpu" for t in ms)
    exp = oracle_mod.compute_dmsc(img, 0.1)
    assert diff_fields(list(ms), exp) == []


@pytest.mark.parametrize("shape", [(1000, 1024), (333, 518), (40, 64)])
@pytest.mark.parametrize("dual", [False, True])
def test_pinned_cpu_input_uploaded_in_bands(shape, dual):
    """A pinned CPU image is uploaded by the library in bands of rows that
    overlap the gradient (dmsc_b200_set_host_input): every output equals the
    call on the same image already on the device. Widths that are multiples
    of 4 take the banded persistent gradient (1000 rows: 8 bands; 40 rows:
    fewer tile rows than bands); 518 columns take the one-copy fallback."""
    from dmsc_b200 import compute_dmsc
    from dmsc_b200.synthetic import field_256_bumps

    g = torch.Generator().manual_seed(5)
    base = field_256_bumps(seed=11)
    img = torch.nn.functional.interpolate(base[None, None], size=shape, mode="bilinear", align_corners=False)[0, 0]
    img = (img + 0.01 * torch.randn(shape, generator=g)).contiguous()
    host = img.pin_memory()
    assert host.is_pinned()
    exp = compute_dmsc(img.cuda(), 0.02, is_dual=dual)
    got = compute_dmsc(host, 0.02, is_dual=dual)
    assert all(t.device.type == "cpu" for t in got)
    assert diff_fields(list(got), [t.cpu() for t in exp]) == []
    # the registration covers one call: the next device call is unaffected
    again = compute_dmsc(img.cuda(), 0.02, is_dual=dual)
    assert diff_fields([t.cpu() for t in again], [t.cpu() for t in exp]) == []


def test_output_devices():
    from dmsc_b200 import compute_dmsc

    ms = compute_dmsc(torch.randn((8, 8), device="cuda"), 0.1)
    assert ms.shape.device.type == "cpu"
    assert all(t.device.type == "cuda" for f, t in zip(FIELDS, ms) if f != "shape")


@pytest.mark.parametrize("value", [0.0, float("inf"), float("-inf"), float("nan")])
def test_constant_fields(oracle_mod, value):
    from dmsc_b200 import compute_dmsc

    field = torch.full((6, 5), value)
    first = compute_dmsc(field.cuda(), 0.0)
    second = compute_dmsc(field.cuda(), 0.0)
    assert diff_fields(list(first), list(second)) == []
    assert diff_fields(list(first), oracle_mod.compute_dmsc(field, 0.0)) == []


def test_too_large_raises():
    from dmsc_b200 import compute_dmsc

    img = torch.zeros((1, 1), device="cuda").expand(23170, 23170)
    with pytest.raises(RuntimeError, match="too large"):
        compute_dmsc(img, 0.0)


@pytest.mark.parametrize("dual,thr", [(False, 0.0), (False, 0.05), (True, 0.0), (True, 0.05)])
def test_full_size_4096(oracle_mod, dual, thr):
    """The headline 4096 x 4096 bump workload (2000 bumps, sigma U[4, 64],
    N(0, 0.02^2) noise), all four (orientation, threshold) variants."""
    from dmsc_b200.synthetic import field_4096_bumps

    img = field_4096_bumps(seed=1234)
    got = gpu_run(img, thr, [True] * 5, dual)
    exp = oracle_mod.run(img, thr, True, dual, True, True, True, True)
    assert diff_fields(got, exp) == []


def test_uniform_2048(oracle_mod):
    """i.i.d. U[0, 1) at 2048^2, the density of the 16384^2 worst case: at
    threshold 0 every output bit for bit; at 0.5 the simplified ridges grow
    past int32 offsets (7e9 cells already at 1024^2), where the reference's
    offsets go negative and it fails, so the GPU must raise, and without arcs
    every other output must match."""
    from dmsc_b200.synthetic import field_uniform

    img = field_uniform(2048, seed=99)
    exp = oracle_mod.run(img, 0.0, True, False, True, True, True, True)
    assert diff_fields(gpu_run(img, 0.0, [True] * 5, False), exp) == []
    exp = oracle_mod.run(img, 0.5, True, False, False, False, True, True)
    assert diff_fields(gpu_run(img, 0.5, [True, False, False, True, True], False), exp) == []
    with pytest.raises(RuntimeError, match="exceeds int32 offsets"):
        oracle_mod.run(img, 0.5, True, False, True, True, True, True)
    with pytest.raises(RuntimeError, match="exceeds int32 offsets"):
        gpu_run(img, 0.5, [True] * 5, False)
    # the context stays usable after the overflow
    assert diff_fields(gpu_run(img, 0.0, [True] * 5, False), oracle_mod.run(img, 0.0, True, False, True, True, True,
                                                                          True)) == []


def test_uniform_512_heavy_cancellation(oracle_mod):
    """U[0, 1) at 512^2 and threshold 0.5: almost every pair cancels and the
    ridges merge into 2.7e8 cells, just inside int32 offsets."""
    from dmsc_b200.synthetic import field_uniform

    img = field_uniform(512, seed=1234)
    exp = oracle_mod.run(img, 0.5, True, False, True, True, True, True)
    got = gpu_run(img, 0.5, [True] * 5, False)
    assert diff_fields(got, exp) == []


@pytest.mark.parametrize("dual", ["primal", "dual"])
@pytest.mark.parametrize("flt,thr", [("raw", -1.0), ("flt", 0.15)])
def test_reference_format_fixtures(dual, flt, thr):
    """The regenerated fixtures in the reference's own torch.save format
    (tests/golden/reference_format), every field bit for bit."""
    import os

    from dmsc_b200 import compute_dmsc

    d = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_format")
    img = torch.load(os.path.join(d, "landscape_32x32.pt"))
    gt = torch.load(os.path.join(d, f"ms_st_{dual}_{flt}.pt"), weights_only=False)
    ms = compute_dmsc(img.cuda(), thr, return_gradient=True, is_dual=dual == "dual")
    assert diff_fields([getattr(ms, k) for k in FIELDS], [gt[k] for k in FIELDS]) == []
