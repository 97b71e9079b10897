"""dmsc_b200: the ``compute_dmsc`` path of thierry-sousbie/dmsc on NVIDIA B200.

Drop-in surface of the reference package (dmsc/__init__.py:1-4):
``compute_dmsc``, ``MSComplex`` and ``generate_noisy_landscape``. The
discrete gradient, critical cells, arcs, persistence pairing, cancellation
replay and basin/peak labels all run as CUDA kernels (sm_100a) behind the C ABI
in ``include/dmsc_b200.h``.
"""

from .dmsc import MSComplex, compute_dmsc, compute_dmsc_batched, extract_dmsc
from .synthetic import generate_noisy_landscape

__all__ = ["compute_dmsc", "compute_dmsc_batched", "generate_noisy_landscape", "MSComplex", "extract_dmsc"]
