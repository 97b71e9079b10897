"""Seeded synthetic scalar fields.

``generate_noisy_landscape`` keeps the reference helper's signature and field
(dmsc/synthetic.py:4-31: two Gaussian peaks, two Gaussian valleys, an optional
extra peak with a slope, plus uniform noise). The other generators build the
benchmark workloads: sums of Gaussian bumps ``a * exp(-r^2 / (2 sigma^2))``
with centres uniform over the image, amplitude ``a ~ U[-amp, amp]`` and
``sigma ~ U[sigma_lo, sigma_hi]`` pixels, plus i.i.d. Gaussian noise; and
i.i.d. uniform [0, 1) fields.
"""

from __future__ import annotations

import math

import torch


def generate_noisy_landscape(H=20, W=20, with_loop=False, z_scale=1.0, noise_scale=0.1):
    """Landscape with noise for persistence tests (dmsc/synthetic.py:4-31)."""
    y, x = torch.meshgrid(torch.linspace(-2, 2, H), torch.linspace(-2, 2, W), indexing="ij")
    z = (torch.exp(-((x - 1) ** 2 + y ** 2) / 0.5) + torch.exp(-((x + 1) ** 2 + y ** 2) / 0.5)
         - 0.5 * torch.exp(-(x ** 2 + (y - 1) ** 2) / 0.5) - 1.0 * torch.exp(-(x ** 2 + (y + 1) ** 2) / 0.5))
    if with_loop:
        z += 1.0 * torch.exp(-((x ** 2 + (y + 1) ** 2) ** 3) / 0.5) - y / 4
    noise = torch.rand(H, W) - 0.5
    return (z * z_scale + noise * noise_scale).to(torch.float32)


def bump_field(H: int, W: int, n_bumps: int, sigma_lo: float, sigma_hi: float, noise: float, seed: int,
               amp: float = 1.0, device="cpu") -> torch.Tensor:
    """Sum of ``n_bumps`` Gaussian bumps plus N(0, noise^2) noise, float32.

    Bump parameters and noise come from a CPU ``torch.Generator`` seeded with
    ``seed``; each bump is accumulated over a +-4 sigma window.
    """
    g = torch.Generator().manual_seed(seed)
    cy = torch.rand(n_bumps, generator=g, dtype=torch.float64) * H
    cx = torch.rand(n_bumps, generator=g, dtype=torch.float64) * W
    a = (torch.rand(n_bumps, generator=g, dtype=torch.float64) * 2 - 1) * amp
    s = torch.rand(n_bumps, generator=g, dtype=torch.float64) * (sigma_hi - sigma_lo) + sigma_lo
    z = torch.zeros(H, W, dtype=torch.float32, device=device)
    ys = torch.arange(H, dtype=torch.float32, device=device)
    xs = torch.arange(W, dtype=torch.float32, device=device)
    for i in range(n_bumps):
        si, yi, xi = float(s[i]), float(cy[i]), float(cx[i])
        r = int(math.ceil(4 * si)) + 1
        y0, y1 = max(0, int(yi) - r), min(H, int(yi) + r + 1)
        x0, x1 = max(0, int(xi) - r), min(W, int(xi) + r + 1)
        if y0 >= y1 or x0 >= x1:
            continue
        dy = (ys[y0:y1] - yi) ** 2
        dx = (xs[x0:x1] - xi) ** 2
        z[y0:y1, x0:x1] += float(a[i]) * torch.exp(-(dy[:, None] + dx[None, :]) / (2 * si * si))
    z += (torch.randn(H, W, generator=g) * noise).to(device)
    return z


def uniform_field(H: int, W: int, seed: int, device="cpu") -> torch.Tensor:
    """i.i.d. uniform [0, 1) float32 field from a seeded CPU generator."""
    g = torch.Generator().manual_seed(seed)
    return torch.rand(H, W, generator=g).to(device)


# Benchmark workloads (sizes and distributions of the headline configurations).
def field_256_bumps(seed: int = 1234, device="cpu"):
    """256 x 256, 24 bumps, sigma U[8, 32], noise N(0, 0.05^2)."""
    return bump_field(256, 256, 24, 8.0, 32.0, 0.05, seed, device=device)


def field_4096_bumps(seed: int = 1234, device="cpu", size: int = 4096):
    """4096 x 4096, 2000 bumps, sigma U[4, 64], noise N(0, 0.02^2); ``size``
    scales the image with the bump count proportional to the area."""
    n = max(1, int(round(2000 * (size / 4096) ** 2)))
    return bump_field(size, size, n, 4.0, 64.0, 0.02, seed, device=device)


def field_uniform(size: int = 16384, seed: int = 1234, device="cpu"):
    """size x size i.i.d. uniform [0, 1) field."""
    return uniform_field(size, size, seed, device=device)


def batch_uneven(n: int = 512, seed: int = 1234, lo: int = 64, hi: int = 2048, device="cpu"):
    """``n`` images with H and W log-uniform in [lo, hi], bump count
    ceil(area / 8000), sigma U[4, 32], noise N(0, 0.03^2); per-image threshold
    U[0.02, 0.2] and is_dual ~ Bernoulli(0.5). Returns (images, thresholds, duals)."""
    g = torch.Generator().manual_seed(seed)
    imgs, thr, dual = [], [], []
    for i in range(n):
        h = int(round(math.exp(math.log(lo) + float(torch.rand(1, generator=g)) * (math.log(hi) - math.log(lo)))))
        w = int(round(math.exp(math.log(lo) + float(torch.rand(1, generator=g)) * (math.log(hi) - math.log(lo)))))
        nb = max(1, math.ceil(h * w / 8000))
        imgs.append(bump_field(h, w, nb, 4.0, 32.0, 0.03, seed * 7919 + i, device=device))
        thr.append(0.02 + 0.18 * float(torch.rand(1, generator=g)))
        dual.append(bool(torch.rand(1, generator=g) < 0.5))
    return imgs, thr, dual
