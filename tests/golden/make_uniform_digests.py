"""Digests of the reference CPU path's outputs on the worst-case field.

The worst-case configuration is one size x size i.i.d. U[0, 1) float32 field
(``dmsc_b200.synthetic.field_uniform(size, seed=1234)``, a CPU generator, so
the same bits on every machine), primal, full outputs, at persistence
thresholds 0 and 0.5. Its outputs are several GB, so only their SHA-256
digests are kept (tests/golden/uniform<size>_digests.json); bench.py checks
the GPU's outputs against them. At threshold 0.5 the reference's simplified
arcs overflow its int32 offsets (arcs_simplification.hxx:150-155) and the
call fails: that message is recorded, and the call without arcs
(trace_max_arcs = trace_min_arcs = False) is digested instead.

Runs the reference built by ``python oracle/build_ref.py --variant ordered``
(all threads, single-thread output order) or the serial build. Needs about
60 GB of host memory at 16384^2.

Usage: ``python tests/golden/make_uniform_digests.py [--size 16384] [--threads N]``.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import resource
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
FIELDS = (
    "shape max_pts min_pts sad_pts e_max e_min p_max p_min ppairs_max ppairs_min grad_indices "
    "peaks ridges ridge_offsets ridge_arc_offsets basins valleys valley_offsets valley_arc_offsets"
).split()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=16384)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=None)
    ap.add_argument("--only", default=None, help="comma-separated run keys (0.0, 0.5_noarcs, 0.5)")
    args = ap.parse_args()
    for sub in ("ordered", ""):
        d = os.path.join(ROOT, "oracle", "_ref", sub) if sub else os.path.join(ROOT, "oracle", "_ref")
        if os.path.exists(os.path.join(d, "dmsc_cpu.so")):
            sys.path.insert(0, d)
            build = sub or "serial"
            break
    else:
        sys.exit("reference checker not built (python oracle/build_ref.py --variant ordered)")
    sys.path.insert(0, ROOT)
    import torch
    import dmsc_cpu

    from dmsc_b200.synthetic import field_uniform

    torch.set_num_threads(args.threads)
    out = args.out or os.path.join(HERE, f"uniform{args.size}_digests.json")
    res = json.load(open(out)) if os.path.exists(out) else {}
    img = field_uniform(args.size, seed=1234)
    res.update({"size": args.size, "seed": 1234, "input_sha256": hashlib.sha256(img.numpy().tobytes()).hexdigest(),
                "reference_build": build, "threads": args.threads})
    runs = [("0.0", 0.0, True), ("0.5_noarcs", 0.5, False), ("0.5", 0.5, True)]
    only = set(args.only.split(",")) if args.only else None
    for key, thr, arcs in runs:
        if only and key not in only:
            continue
        t0 = time.perf_counter()
        try:
            r = dmsc_cpu.extract_dmsc(img, thr, True, False, arcs, arcs, True, True)
            ent = {"seconds": time.perf_counter() - t0, "fields": {}}
            for i, n in enumerate(FIELDS):
                a = r[i].contiguous().numpy()
                ent["fields"][n] = {"shape": list(a.shape), "dtype": str(a.dtype),
                                    "sha256": hashlib.sha256(a.tobytes()).hexdigest()}
            del r
        except Exception as e:  # the reference's own failure, recorded verbatim
            ent = {"seconds": time.perf_counter() - t0, "error": f"{type(e).__name__}: {e}"}
        ent["max_rss_gb"] = resource.getrusage(resource.RUSAGE_SELF).ru_maxrss / 1e6
        res[key] = ent
        print(key, {k: v for k, v in ent.items() if k != "fields"}, flush=True)
        with open(out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
