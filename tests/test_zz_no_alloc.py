"""The allocation-free entry point dmsc_b200_critical_cells_static.

It serves callers that cannot allocate device memory while they call us (for
instance code recording a CUDA graph, or a host framework that hands out only
input and output buffers): it works from a fixed static scratch array of the
library. This test calls it through the C ABI, twice in a row, and checks its
gradient and critical-cell lists against the regular two-phase entry point at
threshold -1 (no cancellation, so every critical cell survives): the gradient
and the extremum lists bit for bit, the saddles as a set (the regular entry
lists them in sweep order, this one in ascending cell order).
This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _static_call(lib, img, dual):
    H, W = img.shape
    dev = img.device
    i32 = dict(dtype=torch.int32, device=dev)
    grad = torch.full((4 * (H + 1) * (W + 1),), -7, **i32)
    mins = torch.full((H * W,), -7, **i32)
    sads = torch.full((H * (W + 1) + (H + 1) * W,), -7, **i32)
    maxs = torch.full(((H + 1) * (W + 1),), -7, **i32)
    counts = torch.zeros(3, **i32)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.dmsc_b200_critical_cells_static(
        ctypes.c_void_p(img.data_ptr()), H, W, 1 if dual else 0, ctypes.c_void_p(grad.data_ptr()),
        ctypes.c_void_p(mins.data_ptr()), ctypes.c_void_p(sads.data_ptr()), ctypes.c_void_p(maxs.data_ptr()),
        ctypes.c_void_p(counts.data_ptr()), ctypes.c_void_p(stream))
    assert rc == 0, lib.dmsc_b200_error_string(rc)
    torch.cuda.synchronize()
    nmin, nsad, nmax = (int(v) for v in counts.cpu())
    return grad.cpu(), mins[:nmin].cpu(), sads[:nsad].cpu(), maxs[:nmax].cpu()


@pytest.mark.parametrize("dual", [False, True])
def test_static_matches_regular_entry(dual):
    from dmsc_b200 import _lib, extract_dmsc
    from dmsc_b200.synthetic import field_256_bumps

    lib = _lib.load()
    for k, img in enumerate([field_256_bumps(seed=21).cuda(),
                             torch.from_numpy(np.random.default_rng(5).integers(0, 3, (97, 130)).astype(np.float32)).cuda()]):
        ref = extract_dmsc(img, -1.0, True, dual, False, False, False, False)
        # maxima are faces in the primal and vertices in the dual (cpu/workspace.hxx:322-362)
        ref_faces, ref_verts = (ref[2], ref[1]) if dual else (ref[1], ref[2])
        for call in range(2):  # two calls in a row share the static scratch
            grad, mins, sads, maxs = _static_call(lib, img, dual)
            assert torch.equal(grad, ref[10].cpu()), (k, call)
            assert torch.equal(maxs, ref_faces.cpu()), (k, call)
            assert torch.equal(mins, ref_verts.cpu()), (k, call)
            assert torch.equal(sads, torch.sort(ref[3].cpu()).values), (k, call)


def test_static_rejects_oversize():
    from dmsc_b200 import _lib

    lib = _lib.load()
    img = torch.zeros((4096, 4096), device="cuda")
    d = ctypes.c_void_p(img.data_ptr())
    rc = lib.dmsc_b200_critical_cells_static(d, 4096, 4096, 0, d, d, d, d, d, None)
    assert rc == 2  # DMSC_B200_ERR_TOO_LARGE, before touching any buffer


def test_static_largest_accepted_size():
    """1743 x 1743 is the largest square image the 8 MiB scratch takes; its
    scratch ends within a few KB of the array's end."""
    from dmsc_b200 import _lib, extract_dmsc

    lib = _lib.load()
    img = torch.rand((1743, 1743), generator=torch.Generator().manual_seed(17)).cuda()
    ref = extract_dmsc(img, -1.0, True, False, False, False, False, False)
    for call in range(2):
        grad, mins, sads, maxs = _static_call(lib, img, False)
        assert torch.equal(grad, ref[10].cpu()), call
        assert torch.equal(mins, ref[2].cpu()), call
        assert torch.equal(maxs, ref[1].cpu()), call
        assert torch.equal(sads, torch.sort(ref[3].cpu()).values), call


def test_static_rejects_first_size_over():
    from dmsc_b200 import _lib

    lib = _lib.load()
    img = torch.zeros((1744, 1744), device="cuda")
    d = ctypes.c_void_p(img.data_ptr())
    rc = lib.dmsc_b200_critical_cells_static(d, 1744, 1744, 0, d, d, d, d, d, None)
    assert rc == 2  # DMSC_B200_ERR_TOO_LARGE


_SIDE_STREAM_SCRIPT = r"""
import sys
sys.path.insert(0, {root!r})
import torch
from tests.test_zz_no_alloc import _static_call
from dmsc_b200 import _lib, extract_dmsc
from dmsc_b200.synthetic import field_256_bumps
lib = _lib.load()
img = field_256_bumps(seed=23).cuda()
torch.cuda.synchronize()
side = torch.cuda.Stream()
with torch.cuda.stream(side):  # the first call of this process runs on a non-blocking side stream
    grad, mins, sads, maxs = _static_call(lib, img, False)
ref = extract_dmsc(img, -1.0, True, False, False, False, False, False)
assert torch.equal(grad, ref[10].cpu())
assert torch.equal(mins, ref[2].cpu()) and torch.equal(maxs, ref[1].cpu())
assert torch.equal(sads, torch.sort(ref[3].cpu()).values)
print("side-stream first call ok")
"""


def test_static_first_call_on_side_stream():
    """The first call of a process sets up the static arrays (device address,
    face-pairing table); it must be correct when made on a side stream that is
    not ordered after the legacy default stream. Run in a fresh process so the
    call really is the first."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _SIDE_STREAM_SCRIPT.format(root=root)], capture_output=True, text=True,
                       timeout=300, cwd=root)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "side-stream first call ok" in r.stdout
