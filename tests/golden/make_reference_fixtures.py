"""Writes exact fixtures in the reference's own regression format.

The reference's tests/generate_ground_truth.py:10-60 saves ``torch.save``
dicts of 16 MSComplex fields for a 32 x 32 noisy landscape (seed 1780627675,
``generate_noisy_landscape(32, 32, with_loop=True)``), primal and dual, raw
(threshold -1) and simplified (threshold 0.15), all with
``return_gradient=True``; its tests/test_regression.py:119-173 loads them.
Its committed files came from an older build (with a known duplicate-cell bug
and an older landscape generator). This script regenerates them from the
reference's CPU path compiled here (oracle/_ref, one thread), in the same
dict format plus the three fields the old files lack: ``grad_indices``,
``ridge_arc_offsets`` and ``valley_arc_offsets``. The landscape is produced
by ``dmsc_b200.synthetic.generate_noisy_landscape``, the same formula as the
reference's current generator (checked bit for bit by the CPU tests).

Usage: ``python tests/golden/make_reference_fixtures.py`` (needs
``python oracle/build_ref.py`` first). Output: tests/golden/reference_format/.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "reference_format")
SEED = 1780627675
FIELDS = (
    "shape max_pts min_pts sad_pts e_max e_min p_max p_min ppairs_max ppairs_min grad_indices "
    "peaks ridges ridge_offsets ridge_arc_offsets basins valleys valley_offsets valley_arc_offsets"
).split()
# the reference's dict (generate_ground_truth.py:37-55) plus the exact-only fields
KEYS = ("shape max_pts min_pts sad_pts e_max e_min p_max p_min ppairs_max ppairs_min peaks basins ridges "
        "ridge_offsets valleys valley_offsets grad_indices ridge_arc_offsets valley_arc_offsets").split()


def landscape():
    sys.path.insert(0, ROOT)
    from dmsc_b200.synthetic import generate_noisy_landscape

    torch.manual_seed(SEED)
    np.random.seed(SEED)
    return generate_noisy_landscape(32, 32, with_loop=True)


def main():
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import dmsc_cpu  # the reference CPU path, serial TBB stand-in

    torch.set_num_threads(1)
    os.makedirs(OUT, exist_ok=True)
    img = landscape()
    torch.save(img, os.path.join(OUT, "landscape_32x32.pt"))
    for is_dual in (False, True):
        for flt, thr in (("raw", -1.0), ("flt", 0.15)):
            r = dmsc_cpu.extract_dmsc(img, thr, True, is_dual, True, True, True, True)
            ms = dict(zip(FIELDS, (r[i] for i in range(19))))
            d = {k: ms[k].clone() for k in KEYS}
            name = f"ms_st_{'dual' if is_dual else 'primal'}_{flt}.pt"
            torch.save(d, os.path.join(OUT, name))
            print(name, {k: tuple(v.shape) for k, v in d.items()})


if __name__ == "__main__":
    main()
