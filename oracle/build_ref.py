"""Build recipe for the reference checker (test infrastructure only).

Compiles the reference's own CPU path, ``dmsc/csrc/dmsc_cpu.cpp`` and the
headers it includes, straight from the read-only reference checkout into
``oracle/_ref/dmsc_cpu.so``. oneTBB is not installed in this image, so the
serial header shim in ``oracle/tbb_shim`` stands in for it; it runs every TBB
construct in program order, which is the reference's canonical 1-thread order.

The checker is used by the CPU tests to pin the C restatement in
``oracle/dmsc_oracle.c`` and by ``bench.py --impl reference`` as the timed CPU
baseline. Nothing in the product path loads it.

Usage: ``python oracle/build_ref.py [--reference DIR]`` (default: $DMSC_REFERENCE,
else ``../reference`` beside the repository).
"""

from __future__ import annotations

import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")


def reference_dir() -> str:
    """Checkout of the reference: $DMSC_REFERENCE, else a ``reference``
    directory beside this repository."""
    env = os.environ.get("DMSC_REFERENCE")
    if env:
        return env
    return os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")


DEFAULT_REFERENCE = reference_dir()


def _gomp_ldflags() -> list[str]:
    """Link the GNU OpenMP runtime by path: the compiler torch picks may not
    find it on its own search path."""
    for cand in ("/usr/lib/x86_64-linux-gnu/libgomp.so.1", "/usr/lib64/libgomp.so.1"):
        if os.path.exists(cand):
            return [cand]
    return ["-fopenmp"]


# TBB stand-ins: "serial" runs every construct in program order (the
# reference's canonical 1-thread order); "ordered" runs them on all threads
# while keeping that order (oracle/tbb_shim_par). Both builds export the
# module ``dmsc_cpu`` (the reference's own module name), from different
# directories, so a process imports one of them.
SHIMS = {"serial": "tbb_shim", "ordered": "tbb_shim_par"}


def out_dir(variant: str = "serial") -> str:
    return OUT if variant == "serial" else os.path.join(OUT, variant)


def build(reference: str = DEFAULT_REFERENCE, verbose: bool = False, variant: str = "serial") -> str | None:
    src = os.path.join(reference, "dmsc", "csrc", "dmsc_cpu.cpp")
    if not os.path.exists(src):
        return None
    from torch.utils.cpp_extension import load

    out = out_dir(variant)
    os.makedirs(out, exist_ok=True)
    load(
        name="dmsc_cpu",
        sources=[src],
        extra_include_paths=[os.path.join(HERE, SHIMS[variant])],
        extra_cflags=["-O3", "-std=c++17", "-fopenmp"],
        extra_ldflags=_gomp_ldflags(),
        build_directory=out,
        verbose=verbose,
        with_cuda=False,
    )
    return os.path.join(out, "dmsc_cpu.so")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("--variant", default="serial", choices=sorted(SHIMS))
    args = ap.parse_args()
    path = build(args.reference, verbose=True, variant=args.variant)
    if path is None:
        print("reference sources not found; checker not built", file=sys.stderr)
        sys.exit(1)
    print(path)
