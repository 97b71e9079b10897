"""The C oracle against the reference: its golden fixtures, the reference's own
fixtures and (when built) the compiled reference on random fields. CPU only."""

import os
import sys

import numpy as np
import pytest
import torch

from oracle import build_ref
from tests.helpers import FIELDS, diff_fields, golden_cases, load_golden

REF_DATA = os.path.join(build_ref.reference_dir(), "tests", "data")
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


def test_oracle_int32_geometry_overflow(oracle_mod):
    """U[0, 1) at 1024^2 with threshold 0.5: the simplified ridges would hold
    about 7e9 cells. The reference's int32 offsets go negative there and the
    call fails (arcs_simplification.hxx:150-155); the oracle stops with an
    error before allocating, and without arcs it completes."""
    from dmsc_b200.synthetic import field_uniform

    img = field_uniform(1024, seed=1234)
    with pytest.raises(RuntimeError, match="exceeds int32 offsets"):
        oracle_mod.run(img, 0.5, True, False, True, True, True, True)
    out = oracle_mod.run(img, 0.5, True, False, False, False, True, True)
    assert out[12].numel() == 0 and out[16].numel() == 0
    ref = _ref()
    if ref is not None:
        with pytest.raises(RuntimeError, match="negative dimension"):
            ref.extract_dmsc(img, 0.5, True, False, True, True, True, True)
        exp = ref.extract_dmsc(img, 0.5, True, False, False, False, True, True)
        assert diff_fields(out, [exp[i] for i in range(19)]) == []


_ORDERED_SCRIPT = r"""
import sys
sys.path.insert(0, {root!r})
sys.path.insert(0, {ref!r})
import numpy as np
import torch
import dmsc_cpu
from oracle import oracle
from tests.helpers import diff_fields, golden_cases, load_golden
torch.set_num_threads(4)
bad = []
for name, path in golden_cases():
    img, thr, dual, fl, exp = load_golden(path)
    r = dmsc_cpu.extract_dmsc(img, thr, fl[0], dual, fl[1], fl[2], fl[3], fl[4])
    if diff_fields([r[i] for i in range(19)], exp):
        bad.append(name)
rng = np.random.default_rng(13)
for it in range(20):
    H, W = int(rng.integers(50, 160)), int(rng.integers(50, 160))
    img = torch.from_numpy(rng.standard_normal((H, W)).astype(np.float32))
    dual = bool(it % 2)
    r = dmsc_cpu.extract_dmsc(img, 0.1, True, dual, True, True, True, True)
    if diff_fields([r[i] for i in range(19)], oracle.run(img, 0.1, True, dual, True, True, True, True)):
        bad.append(f"random {{it}}")
print("BAD", bad)
"""


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_LIB, "ordered", "dmsc_cpu.so")),
                    reason="ordered reference build not present (oracle/build_ref.py --variant ordered)")
def test_ordered_reference_build_is_bit_identical():
    """The reference built with the order-preserving parallel TBB stand-in
    (the timed CPU baseline) gives, on 4 threads, exactly the single-thread
    outputs: the golden fixtures and the oracle on random fields. A separate
    process, since both builds are the module ``dmsc_cpu``."""
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _ORDERED_SCRIPT.format(root=root, ref=os.path.join(REF_LIB, "ordered"))],
                       capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "BAD []" in r.stdout, r.stdout[-2000:]


REF_FORMAT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_format")


@pytest.mark.parametrize("dual", ["primal", "dual"])
@pytest.mark.parametrize("flt,thr", [("raw", -1.0), ("flt", 0.15)])
def test_reference_format_fixtures_match_oracle(oracle_mod, dual, flt, thr):
    """The regenerated fixtures in the reference's torch.save format
    (tests/golden/make_reference_fixtures.py) hold exactly the oracle's
    outputs on their landscape, every field including grad_indices and the
    arc offsets."""
    img = torch.load(os.path.join(REF_FORMAT, "landscape_32x32.pt"))
    gt = torch.load(os.path.join(REF_FORMAT, f"ms_st_{dual}_{flt}.pt"), weights_only=False)
    got = dict(zip(FIELDS, oracle_mod.run(img, thr, True, dual == "dual", True, True, True, True)))
    assert set(gt) == set(FIELDS)
    for k in FIELDS:
        a, e = got[k], gt[k]
        assert a.dtype == e.dtype and a.shape == e.shape, k
        assert torch.equal(a.view(torch.int32) if a.is_floating_point() else a,
                           e.view(torch.int32) if e.is_floating_point() else e), k


def _reference_module(rel, name):
    path = os.path.join(build_ref.reference_dir(), rel)
    if not os.path.exists(path):
        return None
    import importlib.util

    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    try:
        spec.loader.exec_module(mod)
    except Exception:
        return None
    return mod


def test_reference_format_landscape_is_the_reference_generator():
    """The fixtures' landscape is the reference's current generator
    (dmsc/synthetic.py:4-31) at the seed of generate_ground_truth.py."""
    ref = _reference_module(os.path.join("dmsc", "synthetic.py"), "_ref_synthetic")
    if ref is None:
        pytest.skip("reference sources not present")
    torch.manual_seed(1780627675)
    np.random.seed(1780627675)
    exp = ref.generate_noisy_landscape(32, 32, with_loop=True)
    img = torch.load(os.path.join(REF_FORMAT, "landscape_32x32.pt"))
    assert torch.equal(img.view(torch.int32), exp.view(torch.int32))


def test_reference_regression_checks_pass_on_fixtures(oracle_mod):
    """The reference's own regression comparison
    (tests/test_regression.py:20-116, assert_mscomplex_equivalence), run
    against the regenerated fixtures for the outputs of every flag subset the
    regression test uses."""
    import itertools
    import sys as _sys
    import types

    # the module imports dmsc at top level; give it a stub so only its
    # comparison function is used
    stub = "dmsc" not in _sys.modules
    if stub:
        _sys.modules["dmsc"] = types.SimpleNamespace(compute_dmsc=None)
    try:
        mod = _reference_module(os.path.join("tests", "test_regression.py"), "_ref_regression")
    finally:
        if stub:
            del _sys.modules["dmsc"]
    if mod is None:
        pytest.skip("reference tests not present")
    from dmsc_b200.dmsc import MSComplex

    img = torch.load(os.path.join(REF_FORMAT, "landscape_32x32.pt"))
    for dual, (flt, thr) in itertools.product((False, True), (("raw", -1.0), ("flt", 0.15))):
        gt = torch.load(os.path.join(REF_FORMAT, f"ms_st_{'dual' if dual else 'primal'}_{flt}.pt"),
                        weights_only=False)
        for tv, tr, tp, tb in itertools.product((True, False), repeat=4):
            out = oracle_mod.run(img, thr, flt == "raw", dual, tr, tv, tp, tb)
            mod.assert_mscomplex_equivalence(gt, MSComplex(*out), tv, tr, tp, tb)
