"""The gradient kernel's pairing-word encoding and per-index gather, run on the
host (tests/native/gradient_words_host.cu compiles the device functions of
dmsc_b200/csrc/gradient.cuh for the CPU), against the oracle's gradient
(cpu/gradient.hxx:19-196): every slot, and the criticality bits and flow codes
derived from it. CPU only; needs nvcc, skipped without it."""

import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "gradient_words_host.cu")
OUT = os.path.join(ROOT, "tests", "_build", "gradient_words_host.so")
DEPS = [SRC, os.path.join(ROOT, "dmsc_b200", "csrc", "gradient.cuh"), os.path.join(ROOT, "dmsc_b200", "csrc",
                                                                                  "common.cuh")]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else shutil.which("nvcc")


@pytest.fixture(scope="module")
def harness():
    nvcc = _nvcc()
    if not nvcc:
        pytest.skip("nvcc not available")
    if not os.path.exists(OUT) or any(os.path.getmtime(d) > os.path.getmtime(OUT) for d in DEPS):
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-Xcompiler",
                               "-fPIC", "-shared", "--expt-relaxed-constexpr", "-o", OUT + ".tmp", SRC])
        os.replace(OUT + ".tmp", OUT)
    lib = ctypes.CDLL(OUT)
    lib.gradient_words_host.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p]
    return lib


def _host(lib, img, dual):
    a = np.ascontiguousarray(img, dtype=np.float32)
    H, W = a.shape
    n = (H + 1) * (W + 1)
    grad = np.empty(4 * n, np.int32)
    mask = np.empty(n, np.uint8)
    flow = np.empty(n, np.uint8)
    lib.gradient_words_host(a.ctypes.data, H, W, int(dual), grad.ctypes.data, mask.ctypes.data, flow.ctypes.data)
    return grad, mask, flow


def _expected_mask_flow(grad, H, W):
    Nx = W + 1
    g = grad.reshape(H + 1, W + 1, 4)
    iy, ix = np.mgrid[0:H + 1, 0:W + 1]
    b = iy * Nx + ix
    valid = np.stack([(iy < H) & (ix < W), iy < H, ix < W, np.ones_like(iy, bool)], -1)
    crit = valid & (g == -1)
    mask = (crit * (1 << np.arange(4))).sum(-1).astype(np.uint8)
    s0, s3 = g[..., 0], g[..., 3]
    vflow = np.select([s0 == 1 + 4 * b, s0 == 1 + 4 * (b + 1), s0 == 2 + 4 * b, s0 == 2 + 4 * (b + Nx)], [1, 2, 3, 4],
                      0)
    eidx = s3 >> 2
    ffl = np.where(s3 < 0, 0, np.where((s3 & 3) == 1, np.where(eidx == b, 4, 3), np.where(eidx == b, 2, 1)))
    fl = vflow | (crit[..., 1] << 3) | (ffl << 4) | (crit[..., 2] << 7)
    return mask.reshape(-1), fl.astype(np.uint8).reshape(-1)


def _fields(rng):
    for it in range(300):
        H, W = int(rng.integers(1, 30)), int(rng.integers(1, 30))
        kind = it % 5
        if kind == 0:
            a = rng.standard_normal((H, W))
        elif kind == 1:
            a = rng.integers(0, 3, (H, W))
        elif kind == 2:
            a = rng.integers(0, 64, (H, W)) / 64.0
        elif kind == 3:
            a = np.full((H, W), rng.choice([0.0, -0.0, np.inf, -np.inf, np.nan]))
        else:
            a = np.where(rng.random((H, W)) < 0.5, 0.0, -0.0)
        yield a.astype(np.float32)


def test_words_match_oracle_gradient(harness, oracle_mod):
    rng = np.random.default_rng(3)
    for img in _fields(rng):
        for dual in (False, True):
            grad, mask, flow = _host(harness, img, dual)
            exp = oracle_mod.run(torch.from_numpy(img), 0.0, True, dual)[10].numpy()
            assert np.array_equal(grad, exp), (img.shape, dual)
            em, ef = _expected_mask_flow(exp, *img.shape)
            assert np.array_equal(mask, em), (img.shape, dual)
            assert np.array_equal(flow, ef), (img.shape, dual)


def test_words_match_oracle_on_bumps(harness, oracle_mod):
    from dmsc_b200.synthetic import field_256_bumps

    img = field_256_bumps(seed=9).numpy()
    for dual in (False, True):
        grad, _, _ = _host(harness, img, dual)
        assert np.array_equal(grad, oracle_mod.run(torch.from_numpy(img), 0.1, True, dual)[10].numpy())
