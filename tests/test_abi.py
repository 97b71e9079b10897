"""Host-side checks that need no GPU: the C-ABI library loads and exports every
symbol the header declares; the Python boundary raises the reference's errors
before touching the device."""

import ctypes
import os
import re

import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "dmsc_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|long long|const char\*)\s+(dmsc_b200_\w+)\s*\(", src, re.M)))


def test_library_exports_header_symbols():
    from dmsc_b200 import _lib

    lib = _lib.load()
    names = header_functions()
    assert set(names) == set(_lib.EXPORTS)
    for n in names:
        assert hasattr(lib, n), n


def test_error_strings_without_device():
    from dmsc_b200 import _lib

    lib = _lib.load()
    for code in range(7):
        assert lib.dmsc_b200_error_string(code)
    assert lib.dmsc_b200_last_error(None) == b""


def test_extract_rejects_null_context():
    from dmsc_b200 import _lib

    lib = _lib.load()
    assert lib.dmsc_b200_extract(None, None, 1, 1, ctypes.c_float(0.0), 0, None, None, None, None, None) == 1


@pytest.mark.parametrize("shape", [(0, 4), (4, 0), (0, 4, 4)])
def test_rejects_empty_dimensions(shape):
    from dmsc_b200 import compute_dmsc

    with pytest.raises(ValueError, match="non-empty"):
        compute_dmsc(torch.empty(shape), 0.0)


@pytest.mark.parametrize("dtype", [torch.float16, torch.float64, torch.int32, torch.int64])
def test_rejects_unsupported_dtype(dtype):
    from dmsc_b200 import compute_dmsc

    with pytest.raises(TypeError, match="float32"):
        compute_dmsc(torch.zeros((4, 4), dtype=dtype), 0.0)


def test_rejects_bad_rank():
    from dmsc_b200 import compute_dmsc

    with pytest.raises(ValueError, match="2D"):
        compute_dmsc(torch.zeros(4), 0.0)


def test_mscomplex_helpers():
    from dmsc_b200 import MSComplex

    z = torch.zeros(0, dtype=torch.int32)
    ms = MSComplex(torch.tensor([2, 3], dtype=torch.int32), *([z] * 18))
    assert ms.Nx == 4
    cells = torch.tensor([0, 1, 2, 3, 4 * 5 + 3], dtype=torch.int32)
    yx = ms.to_coordinates_yx(cells)
    assert yx.tolist() == [[0.0, 0.0], [0.0, -0.5], [-0.5, 0.0], [-0.5, -0.5], [0.5, 0.5]]
    assert ms.to_coordinates_yx(cells, staggered=False).tolist() == [[0, 0]] * 4 + [[1, 1]]
    assert len(ms) == 19 and len(list(ms)) == 19
