"""Differentiable persistence values (dmsc_b200.autograd): forward values
equal compute_dmsc's, pixel pairs equal the oracle's pairs, the backward
kernel equals a plain-torch gradient built from the oracle's pairs and FP64
central finite differences, and is deterministic."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def tie_free_field(H, W, seed, bumps=None, check=True):
    """Bump + noise field plus 1e-6 * rank / N for a random permutation rank.
    At large N that step is below float32 resolution, so ties are checked on
    the array actually tested (``check``)."""
    from dmsc_b200.synthetic import bump_field

    nb = bumps if bumps is not None else max(1, round(200 * H * W / 512**2))
    f = bump_field(H, W, nb, 4.0, 32.0, 0.05, seed)
    g = torch.Generator().manual_seed(seed + 1)
    rank = torch.randperm(H * W, generator=g).reshape(H, W).float()
    f = f + 1e-6 * rank / (H * W)
    if check:
        assert torch.unique(f).numel() == H * W
    return f


def value_pixel(img, cell, dual):
    """Image-local value pixel of a cell: its highest (dual: lowest) vertex
    under the (value, pixel id) order (cell_compare.hxx:33-87)."""
    H, W = img.shape
    Nx = W + 1
    t, idx = cell & 3, cell >> 2
    y, x = divmod(idx, Nx)
    if t == 0:
        c = [(y, x)]
    elif t == 1:
        c = [(y, x + dx) for dx in (-1, 0) if 0 <= x + dx < W]
    elif t == 2:
        c = [(y + dy, x) for dy in (-1, 0) if 0 <= y + dy < H]
    else:
        c = [(y + dy, x + dx) for dy in (-1, 0) for dx in (-1, 0) if 0 <= y + dy < H and 0 <= x + dx < W]
    keys = [(float(img[a, b]), a * W + b) for a, b in c]
    best = min(keys) if dual else max(keys)
    return best[1]


def oracle_pairs(oracle_mod, img, thr, dual):
    """Per public side, per sad_pts entry: (plus, minus) pixels from the
    oracle's own saddle-extremum pairs."""
    main, dbg = oracle_mod.run(img, thr, False, dual, debug=True)
    sad_pts = main[3].numpy()
    crit_sad = dbg["crit_saddles"].numpy()
    pos = {int(c): k for k, c in enumerate(crit_sad)}
    a = img.numpy()
    res = {}
    # internal vertex side = public min in the primal, public max in the dual
    for pub, internal, vertex_side in (("min", "pair_min", True), ("max", "pair_max", False)):
        if dual:
            internal, vertex_side = ("pair_max", False) if pub == "min" else ("pair_min", True)
        pairs = dbg[internal].numpy()
        plus, minus = [], []
        for c in sad_pts:
            e = int(pairs[pos[int(c)]])
            if e < 0:
                plus.append(-1)
                minus.append(-1)
                continue
            sp, ep = value_pixel(a, int(c), dual), value_pixel(a, e, dual)
            saddle_plus = vertex_side != dual
            plus.append(sp if saddle_plus else ep)
            minus.append(ep if saddle_plus else sp)
        res[pub] = (np.array(plus, dtype=np.int32), np.array(minus, dtype=np.int32))
    return main, res


@pytest.mark.parametrize("dual", [False, True])
@pytest.mark.parametrize("thr", [-1.0, 0.05])
def test_values_and_pixels_match(oracle_mod, dual, thr):
    from dmsc_b200 import compute_dmsc
    from dmsc_b200.autograd import persistence_pairs

    img = tie_free_field(96, 80, seed=3)
    ms = compute_dmsc(img.cuda(), thr, is_dual=dual)
    pp = persistence_pairs(img.cuda(), thr, is_dual=dual)
    p = pp.persistence.detach()
    side = pp.side.cpu()
    exp_p = torch.cat([ms.p_min.cpu(), ms.p_max.cpu()])
    assert torch.equal(p.cpu().view(torch.int32), exp_p.view(torch.int32))
    assert torch.equal(pp.ppairs.cpu(), torch.cat([ms.ppairs_min.cpu(), ms.ppairs_max.cpu()]))
    assert int((side == 0).sum()) == ms.p_min.numel()
    # p is the float32 difference of the two pixels, bit for bit
    plus, minus = pp.plus_pixel.cpu().long(), pp.minus_pixel.cpu().long()
    ok = plus >= 0
    flat = img.reshape(-1)
    diff = flat[plus[ok]] - flat[minus[ok]]
    assert torch.equal(diff.view(torch.int32), p.cpu()[ok].view(torch.int32))
    assert torch.all(p.cpu()[~ok] == -1.0)
    # the pixel pairs are the oracle's pairs
    _, ref = oracle_pairs(oracle_mod, img, thr, dual)
    n_min = ms.p_min.numel()
    assert np.array_equal(plus[:n_min].numpy(), ref["min"][0]) and np.array_equal(minus[:n_min].numpy(), ref["min"][1])
    assert np.array_equal(plus[n_min:].numpy(), ref["max"][0]) and np.array_equal(minus[n_min:].numpy(), ref["max"][1])


def _torch_loss_from_pairs(img, plus, minus, ppairs, maxp=0.1):
    flat = img.reshape(-1)
    ok = torch.as_tensor(plus >= 0)
    pl = torch.as_tensor(plus[ok.numpy()]).long()
    mi = torch.as_tensor(minus[ok.numpy()]).long()
    p = flat[pl] - flat[mi]
    keep = (torch.as_tensor(ppairs)[ok] != -1) & (p >= 0) & (p < maxp)
    return (p * p * keep).sum()


@pytest.mark.parametrize("dual", [False, True])
def test_backward_matches_plain_torch_from_oracle_pairs(oracle_mod, dual):
    from dmsc_b200.autograd import topological_loss

    img = tie_free_field(128, 112, seed=9)
    x = img.cuda().requires_grad_(True)
    loss = topological_loss(x, -1.0, 0.1, is_dual=dual)
    loss.backward()
    main, ref = oracle_pairs(oracle_mod, img, -1.0, dual)
    plus = np.concatenate([ref["min"][0], ref["max"][0]])
    minus = np.concatenate([ref["min"][1], ref["max"][1]])
    ppairs = np.concatenate([main[9].numpy(), main[8].numpy()])  # ppairs_min, ppairs_max
    xr = img.clone().requires_grad_(True)
    lr = _torch_loss_from_pairs(xr, plus, minus, ppairs)
    lr.backward()
    assert abs(loss.item() - lr.item()) <= 1e-5 * max(1.0, abs(lr.item()))
    assert torch.allclose(x.grad.cpu(), xr.grad, rtol=1e-5, atol=1e-7)
    assert int((x.grad != 0).sum()) > 0


def test_fp64_finite_differences():
    """Central differences (step 1e-4) of the loss recomputed in FP64 from the
    pairs at the perturbed field, on a 64 x 64 crop; pixels whose pairing or
    loss mask changes within the step are skipped (few on a tie-free field)."""
    from dmsc_b200.autograd import persistence_pairs, topological_loss

    field = tie_free_field(512, 512, seed=21, check=False)
    crop = field[200:264, 300:364].contiguous()
    assert torch.unique(crop).numel() == crop.numel()
    x = crop.cuda().requires_grad_(True)
    topological_loss(x, -1.0, 0.1).backward()
    an = x.grad.double().cpu().reshape(-1)

    def loss64(batch32, batch64):
        pp = persistence_pairs(batch32.cuda(), -1.0)
        p32 = pp.persistence.detach()
        keep = ((pp.ppairs != -1) & (p32 >= 0) & (p32 < 0.1)).cpu()
        img = pp.image.cpu()
        plus, minus = pp.plus_pixel.cpu().long(), pp.minus_pixel.cpu().long()
        ok = plus >= 0
        flat = batch64.reshape(batch64.shape[0], -1)
        p64 = torch.zeros(p32.numel(), dtype=torch.float64)
        p64[ok] = flat[img[ok], plus[ok]] - flat[img[ok], minus[ok]]
        sig = [tuple(t) for t in torch.stack([img, plus, minus, keep.long()], 1)[keep].tolist()]
        out = torch.zeros(batch64.shape[0], dtype=torch.float64).index_add_(0, img, p64 * p64 * keep)
        per_img = [set() for _ in range(batch64.shape[0])]
        for b, a, m, _ in sig:
            per_img[b].add((a, m))
        return out, per_img

    base64 = crop.double()
    _, base_sig = loss64(crop.unsqueeze(0), base64.unsqueeze(0))
    h = 1e-4
    N = crop.numel()
    fd = torch.zeros(N, dtype=torch.float64)
    stable = torch.zeros(N, dtype=torch.bool)
    chunk = 512
    for s in range(0, N, chunk):
        idx = torch.arange(s, min(N, s + chunk))
        k = idx.numel()
        b64 = base64.reshape(1, -1).repeat(2 * k, 1)
        b64[torch.arange(k), idx] += h
        b64[torch.arange(k, 2 * k), idx] -= h
        b64 = b64.reshape(2 * k, *crop.shape)
        b32 = b64.float()
        b64 = b32.double()  # the field the pairing saw, exactly
        L, sigs = loss64(b32, b64)
        steps = (b64.reshape(2 * k, -1)[torch.arange(k), idx] - b64.reshape(2 * k, -1)[torch.arange(k, 2 * k), idx])
        fd[idx] = (L[:k] - L[k:]) / steps
        for j in range(k):
            stable[idx[j]] = sigs[j] == base_sig[0] and sigs[k + j] == base_sig[0]
    assert stable.float().mean() > 0.95
    scale = an.abs().max()
    err = (fd - an)[stable].abs().max()
    assert err <= 1e-5 * scale, (float(err), float(scale))


def test_backward_is_deterministic_and_batch_consistent():
    from dmsc_b200.autograd import persistence_pairs

    imgs = torch.stack([tie_free_field(200, 200, seed=s, check=False) for s in (1, 2, 3)]).cuda()
    grads = []
    for _ in range(2):
        x = imgs.clone().requires_grad_(True)
        pp = persistence_pairs(x, [0.02, -1.0, 0.05], is_dual=[False, True, False])
        w = torch.linspace(0.5, 1.5, pp.persistence.numel(), device="cuda")
        (pp.persistence * w).sum().backward()
        grads.append(x.grad.clone())
    assert torch.equal(grads[0].view(torch.int32), grads[1].view(torch.int32))
    # each image alone gives the same bits (same per-pixel summation order)
    x = imgs.clone().requires_grad_(True)
    pp = persistence_pairs(x, [0.02, -1.0, 0.05], is_dual=[False, True, False])
    g = torch.ones_like(pp.persistence)
    (pp.persistence * g).sum().backward()
    for b, (t, d) in enumerate(((0.02, False), (-1.0, True), (0.05, False))):
        xb = imgs[b].clone().requires_grad_(True)
        persistence_pairs(xb, t, is_dual=d).persistence.sum().backward()
        assert torch.equal(xb.grad.view(torch.int32), x.grad[b].view(torch.int32)), b


def test_scatter_edge_cases():
    from dmsc_b200.autograd import scatter_pair_grads

    dev = "cuda"
    plus = torch.tensor([0, 5, -1, 5, 3], dtype=torch.int32, device=dev)
    minus = torch.tensor([5, 0, -1, 7, 3], dtype=torch.int32, device=dev)
    g = torch.tensor([1.0, 2.0, 100.0, 0.25, 4.0], device=dev)
    out = scatter_pair_grads(plus, minus, g, (2, 4))
    exp = torch.zeros(8)
    for p, m, v in zip(plus.tolist(), minus.tolist(), g.tolist()):
        if p >= 0:
            exp[p] += v
        if m >= 0:
            exp[m] -= v
    assert torch.equal(out.cpu().reshape(-1), exp)
    empty = scatter_pair_grads(plus[:0], minus[:0], g[:0], (3, 3))
    assert torch.equal(empty.cpu(), torch.zeros(3, 3))


def _fd_check(loss_from_pairs, crop, h=1e-4):
    """Gradient of ``loss_from_pairs(p, image, side, ppairs)`` through
    persistence_pairs against FP64 central differences of the same function
    evaluated on FP64 values of the pairs found at each perturbed field;
    pixels whose pairing (or selected set) changes within the step are
    skipped. Returns (max abs error on stable pixels, gradient scale,
    fraction of stable pixels)."""
    from dmsc_b200.autograd import persistence_pairs

    x = crop.cuda().requires_grad_(True)
    pp = persistence_pairs(x, -1.0)
    loss_from_pairs(pp.persistence, pp.image, pp.side, pp.ppairs).sum().backward()
    an = x.grad.double().cpu().reshape(-1)

    def eval64(b32):
        q = persistence_pairs(b32.cuda(), -1.0)
        img, side, ppairs = q.image.cpu(), q.side.cpu(), q.ppairs.cpu()
        plus, minus = q.plus_pixel.cpu().long(), q.minus_pixel.cpu().long()
        ok = plus >= 0
        flat = b32.double().reshape(b32.shape[0], -1)
        p64 = torch.full((plus.numel(),), -1.0, dtype=torch.float64)
        p64[ok] = flat[img[ok], plus[ok]] - flat[img[ok], minus[ok]]
        L = loss_from_pairs(p64, img, side, ppairs, n_images=b32.shape[0])
        # what the losses select: every pair, whether it is under the
        # denoising cut, and the five most persistent pairs of each side
        sig = [set() for _ in range(b32.shape[0])]
        best = {}
        for b, s, a, m, v in zip(img.tolist(), side.tolist(), plus.tolist(), minus.tolist(), p64.tolist()):
            sig[b].add((s, a, m, v < 0.1))
            best.setdefault((b, s), []).append((-v, a, m))
        for (b, s), lst in best.items():
            sig[b].add(("top", s, tuple((a, m) for _, a, m in sorted(lst)[:5])))
        return L, sig

    _, base_sig = eval64(crop.unsqueeze(0))
    N = crop.numel()
    fd = torch.zeros(N, dtype=torch.float64)
    stable = torch.zeros(N, dtype=torch.bool)
    chunk = 512
    base64 = crop.double()
    for s in range(0, N, chunk):
        idx = torch.arange(s, min(N, s + chunk))
        k = idx.numel()
        b64 = base64.reshape(1, -1).repeat(2 * k, 1)
        b64[torch.arange(k), idx] += h
        b64[torch.arange(k, 2 * k), idx] -= h
        b32 = b64.reshape(2 * k, *crop.shape).float()
        L, sigs = eval64(b32)
        b64 = b32.double().reshape(2 * k, -1)
        steps = b64[torch.arange(k), idx] - b64[torch.arange(k, 2 * k), idx]
        fd[idx] = (L[:k] - L[k:]) / steps
        for j in range(k):
            stable[idx[j]] = sigs[j] == base_sig[0] and sigs[k + j] == base_sig[0]
    scale = an.abs().max()
    return float((fd - an)[stable].abs().max()), float(scale), float(stable.float().mean())


@pytest.mark.parametrize("name", ["denoise_min", "denoise_max", "betti_min", "betti_max", "segmentation"])
def test_loss_library_fp64_finite_differences(name):
    """Each loss of dmsc_b200.losses against FP64 central differences (step
    1e-4) on a tie-free 48 x 48 crop, within 1e-5 of the gradient's scale."""
    from dmsc_b200 import losses

    fns = {
        "denoise_min": lambda p, i, s, q, n_images=None: losses.denoising_loss_from_pairs(p, i, s, q, 0.1, "min",
                                                                                            n_images),
        "denoise_max": lambda p, i, s, q, n_images=None: losses.denoising_loss_from_pairs(p, i, s, q, 0.1, "max",
                                                                                            n_images),
        "betti_min": lambda p, i, s, q, n_images=None: losses.betti_loss_from_pairs(p, i, s, q, 3, "min", 1.0,
                                                                                      n_images),
        "betti_max": lambda p, i, s, q, n_images=None: losses.betti_loss_from_pairs(p, i, s, q, 2, "max", 0.5,
                                                                                      n_images),
        "segmentation": lambda p, i, s, q, n_images=None: (
            losses.betti_loss_from_pairs(p, i, s, q, 3, "min", 1.0, n_images)
            + losses.betti_loss_from_pairs(p, i, s, q, 2, "max", 1.0, n_images)),
    }
    field = tie_free_field(512, 512, seed=23, check=False)
    crop = field[100:148, 260:308].contiguous()
    assert torch.unique(crop).numel() == crop.numel()
    err, scale, frac = _fd_check(fns[name], crop)
    assert frac > 0.95
    assert scale > 0
    assert err <= 1e-5 * scale, (err, scale)


def test_loss_library_public_forms_match_pairs():
    """The image-level forms equal their *_from_pairs forms on one forward,
    and segmentation_loss is the sum of the two side losses."""
    from dmsc_b200 import losses
    from dmsc_b200.autograd import persistence_pairs

    x = torch.stack([tie_free_field(96, 96, seed=s, check=False) for s in (4, 5)]).cuda()
    pp = persistence_pairs(x, -1.0)
    a = losses.betti_loss(x, [2, 4], "min", reduction="none")
    b = losses.betti_loss_from_pairs(pp.persistence, pp.image, pp.side, pp.ppairs, [2, 4], "min", 1.0, 2)
    assert torch.equal(a, b)
    s = losses.segmentation_loss(x, n_basins=[2, 4], n_peaks=3, reduction="none")
    c = b + losses.betti_loss_from_pairs(pp.persistence, pp.image, pp.side, pp.ppairs, 3, "max", 1.0, 2)
    assert torch.allclose(s, c)
    d = losses.denoising_loss(x, 0.1, "both")
    from dmsc_b200.autograd import topological_loss
    assert torch.allclose(d, topological_loss(x, -1.0, 0.1))
