"""The C-ABI library loads and exports every entry point of include/bsr_b200.h.

Only host-side functions are called here (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from tests.conftest import ROOT

HEADER = os.path.join(ROOT, "include", "bsr_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(bsrg_\w+)\s*\(", txt)))


def test_header_declares_the_binding():
    from bsr_b200 import _lib
    names = {n for n, _, _ in _lib.SIGNATURES}
    assert set(declared_symbols()) == names


def test_library_exports_every_symbol():
    from bsr_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.fail("libbsrgpu.so not built (run __graft_entry__.build())")
    L = ctypes.CDLL(_lib.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(L, name), name


@pytest.mark.parametrize("grid_type", [0, 1])
def test_mkgrid_host_matches_oracle(grid_type):
    """bsrg_mkgrid (define_grid.f90:86/:213) is host code: bit-identical to the oracle."""
    from bsr_b200.core import define_grid
    from oracle import oracle as O
    args = (8, 2.0, 0.125, 160.0, 160.0) if grid_type == 0 else (8, 2.0, 0.25, 1.0, 40.0)
    a = define_grid(grid_type, *args)
    b = O.mkgrid(grid_type, *args)
    assert (a["ns"], a["ml"], a["me"]) == (b["ns"], b["ml"], b["me"])
    assert np.array_equal(a["t"], b["t"])


def test_error_reporting_without_gpu():
    from bsr_b200._lib import BsrgError, call
    t = np.zeros(4)
    with pytest.raises(BsrgError) as ei:
        call("bsrg_mkgrid", 0, 40, 1.0, 0.1, 1.0, 1.0, t.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 4,
             ctypes.byref(ctypes.c_int()), ctypes.byref(ctypes.c_int()), ctypes.byref(ctypes.c_int()),
             ctypes.byref(ctypes.c_double()))
    assert ei.value.status == -1 and "ks" in str(ei.value)
