"""Loss functions of dmsc_b200.losses on hand-made persistence pairs (CPU,
pure torch): values against a direct per-image computation, gradients
against torch.autograd of that computation."""

import pytest
import torch

from dmsc_b200.losses import betti_loss_from_pairs, denoising_loss_from_pairs


def _pairs(seed):
    g = torch.Generator().manual_seed(seed)
    n = 60
    p = torch.rand(n, generator=g, dtype=torch.float64) * 0.5
    image = torch.sort(torch.randint(0, 3, (n,), generator=g)).values
    side = torch.randint(0, 2, (n,), generator=g).to(torch.int8)
    ppairs = torch.randint(0, 50, (n,), generator=g).to(torch.int32)
    cyc = torch.rand(n, generator=g) < 0.1
    ppairs[cyc] = -1
    p = torch.where(cyc, torch.full_like(p, -1.0), p)
    return p, image, side, ppairs


def _direct_betti(p, image, side, ppairs, k, which, target, B):
    out = []
    for b in range(B):
        sel = [(float(p[i]), i) for i in range(len(p)) if int(image[i]) == b and int(ppairs[i]) != -1
               and float(p[i]) >= 0 and int(side[i]) in which]
        sel.sort(key=lambda t: (-t[0], t[1]))
        kb = k[b] if isinstance(k, (list, tuple)) else k
        tot = 0.0
        for r, (v, _) in enumerate(sel):
            tot += (target - v) ** 2 if r < kb - 1 else v * v
        out.append(tot)
    return torch.tensor(out, dtype=torch.float64)


@pytest.mark.parametrize("side,which", [("min", (0,)), ("max", (1,)), ("both", (0, 1))])
def test_betti_values(side, which):
    for seed in range(5):
        p, image, st, pp = _pairs(seed)
        for k in (1, 2, 4, [1, 3, 5]):
            got = betti_loss_from_pairs(p, image, st, pp, k, side, 0.9, 3)
            exp = _direct_betti(p, image, st, pp, k, which, 0.9, 3)
            assert torch.allclose(got, exp, rtol=1e-12, atol=1e-12), (seed, k)


def test_denoising_values_and_grad():
    p, image, st, pp = _pairs(7)
    p = p.clone().requires_grad_(True)
    got = denoising_loss_from_pairs(p, image, st, pp, 0.2, "min", 3)
    keep = (st == 0) & (pp != -1) & (p.detach() >= 0) & (p.detach() < 0.2)
    exp = torch.zeros(3, dtype=torch.float64).index_add(0, image, (p.detach() ** 2) * keep)
    assert torch.allclose(got.detach(), exp)
    got.sum().backward()
    assert torch.allclose(p.grad, 2 * p.detach() * keep)


def test_betti_gradient():
    p, image, st, pp = _pairs(11)
    p = p.clone().requires_grad_(True)
    betti_loss_from_pairs(p, image, st, pp, 3, "max", 1.0, 3).sum().backward()
    g = p.grad
    p = p.detach()
    # every kept pair gets -2 (1 - p) (top k - 1 of its image) or 2 p; others 0
    for b in range(3):
        idx = [i for i in range(len(p)) if int(image[i]) == b and int(st[i]) == 1 and int(pp[i]) != -1 and
               float(p[i]) >= 0]
        idx.sort(key=lambda i: (-float(p[i]), i))
        for r, i in enumerate(idx):
            v = float(p[i])
            assert abs(float(g[i]) - (-2 * (1 - v) if r < 2 else 2 * v)) < 1e-12
    others = (st != 1) | (pp == -1)
    assert torch.all(g[others] == 0)


def test_argument_errors():
    p, image, st, pp = _pairs(1)
    with pytest.raises(ValueError):
        betti_loss_from_pairs(p, image, st, pp, 0, "min", 1.0, 3)
    with pytest.raises(ValueError):
        betti_loss_from_pairs(p, image, st, pp, [1, 2], "min", 1.0, 3)
    with pytest.raises(ValueError):
        denoising_loss_from_pairs(p, image, st, pp, 0.1, "sideways", 3)
