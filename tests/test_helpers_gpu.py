"""Device-side MSComplex helpers (dmsc/dmsc.py:87-156): to_coordinates_yx,
get_ridge / get_valley (sync-free slices) and their batched forms
get_ridges / get_valleys, against the reference's own slicing semantics
applied to the same tensors on the CPU."""

import pytest
import torch

pytestmark = pytest.mark.gpu


def _ref_slice(pts, off, aoff, i, split):
    # the reference's get_ridge body (dmsc/dmsc.py:132-143) on CPU tensors
    start = off[i]
    end = off[i + 1] if i + 1 < len(off) else len(pts)
    seg = pts[start:end]
    if split:
        s = aoff[i]
        return seg[: s - start], seg[s - start: end - start]
    return seg


@pytest.mark.parametrize("dual", [False, True])
def test_arc_helpers_match_reference_semantics(dual):
    from dmsc_b200 import compute_dmsc
    from dmsc_b200.synthetic import field_256_bumps

    ms = compute_dmsc(field_256_bumps(seed=41).cuda(), 0.05, is_dual=dual)
    n = len(ms.sad_pts)
    assert n > 10
    for name in ("ridge", "valley"):
        pts, off, aoff = (getattr(ms, name + "s").cpu(), getattr(ms, name + "_offsets").cpu(),
                          getattr(ms, name + "_arc_offsets").cpu())
        get = getattr(ms, "get_" + name)
        for i in range(n):
            assert torch.equal(get(i).cpu(), _ref_slice(pts, off, aoff, i, False))
            a, b = get(i, split_arcs=True)
            ea, eb = _ref_slice(pts, off, aoff, i, True)
            assert torch.equal(a.cpu(), ea) and torch.equal(b.cpu(), eb)
        idx = torch.tensor([n - 1, 0, 3, 3, n // 2], device="cuda")
        cells, offs, first = getattr(ms, "get_" + name + "s")(idx)
        for k, i in enumerate(idx.tolist()):
            seg = cells[offs[k]:offs[k + 1]].cpu()
            assert torch.equal(seg, _ref_slice(pts, off, aoff, i, False))
            assert int(first[k]) - int(offs[k]) == int(aoff[i]) - int(off[i])
        empty = getattr(ms, "get_" + name + "s")(torch.empty(0, dtype=torch.int64, device="cuda"))
        assert empty[0].numel() == 0 and empty[1].tolist() == [0]


def test_coordinates_match_reference_formula():
    from dmsc_b200 import compute_dmsc
    from dmsc_b200.synthetic import field_256_bumps

    ms = compute_dmsc(field_256_bumps(seed=42).cuda(), 0.1)
    for cells in (ms.max_pts, ms.min_pts, ms.sad_pts, ms.ridges[:1000]):
        yx = ms.to_coordinates_yx(cells)
        c = cells.cpu().long()
        t, idx = c % 4, c // 4
        y, x = (idx // ms.Nx).float(), (idx % ms.Nx).float()
        y = y - torch.where((t == 2) | (t == 3), 0.5, 0.0)
        x = x - torch.where((t == 1) | (t == 3), 0.5, 0.0)
        assert torch.equal(yx.cpu(), torch.stack([y, x], -1))
        assert yx.device == cells.device
