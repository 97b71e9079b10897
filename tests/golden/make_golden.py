"""Generates the golden fixtures in this folder from the reference itself.

Runs the reference's own CPU path, compiled from the read-only reference
sources by ``oracle/build_ref.py`` into ``oracle/_ref/dmsc_cpu.so``, with one
thread (its canonical output order), on small seeded fields that cover the
edge cases of the path: ties, +-0, constant and non-finite fields, 1-pixel
rows and columns, primal and dual, several thresholds and flag subsets.
Each case is saved as ``<name>.npz`` with the input, the arguments and all 19
outputs of ``extract_dmsc``.

Usage: ``python tests/golden/make_golden.py`` (needs the reference checker).
"""

from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

FIELDS = (
    "shape max_pts min_pts sad_pts e_max e_min p_max p_min ppairs_max ppairs_min grad_indices "
    "peaks ridges ridge_offsets ridge_arc_offsets basins valleys valley_offsets valley_arc_offsets"
).split()


def cases():
    from dmsc_b200.synthetic import bump_field, generate_noisy_landscape

    rng = np.random.default_rng(20261203)
    full = (True, True, True, True, True)  # return_gradient, ridges(max arcs), valleys(min arcs), peaks, basins
    torch.manual_seed(1780627675)
    land = generate_noisy_landscape(32, 32, with_loop=True)
    yield "landscape32_primal_raw", land, -1.0, False, full
    yield "landscape32_primal_flt", land, 0.15, False, full
    yield "landscape32_dual_raw", land, -1.0, True, full
    yield "landscape32_dual_flt", land, 0.15, True, full
    b = bump_field(64, 64, 4, 4.0, 16.0, 0.05, 7)
    for thr in (0.0, 0.05, 0.1):
        for dual in (False, True):
            yield f"bumps64_thr{thr}_{'dual' if dual else 'primal'}", b, thr, dual, full
    b2 = bump_field(96, 80, 6, 4.0, 24.0, 0.03, 11)
    yield "bumps96x80_thr0.1_primal", b2, 0.1, False, full
    yield "bumps96x80_thr0.1_dual_ridges_only", b2, 0.1, True, (False, True, False, True, False)
    yield "bumps96x80_thr0.1_valleys_basins", b2, 0.1, False, (False, False, True, False, True)
    ints = torch.from_numpy(rng.integers(0, 3, (20, 17)).astype(np.float32))
    for thr in (0.0, 1.0):
        for dual in (False, True):
            yield f"ints20x17_thr{thr}_{'dual' if dual else 'primal'}", ints, thr, dual, full
    z = np.zeros((9, 11), np.float32)
    z[rng.random((9, 11)) < 0.5] = -0.0
    z[rng.random((9, 11)) < 0.2] = 1.0
    yield "signed_zeros9x11", torch.from_numpy(z), 0.0, False, full
    for v, nm in ((0.0, "zero"), (float("inf"), "posinf"), (float("-inf"), "neginf"), (float("nan"), "nan")):
        yield f"const6x5_{nm}", torch.full((6, 5), v), 0.0, False, full
    for H, W in ((1, 1), (1, 7), (7, 1), (2, 2), (3, 1), (1, 3)):
        yield f"tiny{H}x{W}", torch.from_numpy(rng.standard_normal((H, W)).astype(np.float32)), 0.1, False, full
        yield f"tiny{H}x{W}_dual", torch.from_numpy(rng.standard_normal((H, W)).astype(np.float32)), 0.1, True, full
    u = torch.from_numpy((rng.integers(0, 1 << 12, (40, 40)) / (1 << 12)).astype(np.float32))
    yield "uniform40_thr0.3", u, 0.3, False, full
    yield "uniform40_thr0_dual", u, 0.0, True, full


def main():
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import dmsc_cpu  # the compiled reference checker

    torch.set_num_threads(1)
    n = 0
    for name, img, thr, dual, fl in cases():
        r = dmsc_cpu.extract_dmsc(img.contiguous(), thr, fl[0], dual, fl[1], fl[2], fl[3], fl[4])
        arrs = {f: r[i].numpy() for i, f in enumerate(FIELDS)}
        np.savez_compressed(os.path.join(HERE, name + ".npz"), image=img.numpy(), threshold=np.float32(thr),
                            is_dual=dual, flags=np.array(fl), **arrs)
        n += 1
    print(f"wrote {n} fixtures")


if __name__ == "__main__":
    main()
