"""bsrg_mrk_cell_noalloc: the R^k table for callers that cannot allocate device memory.

A serving process that has divided all of its HBM among its solves, or a loop
that cannot afford the device-wide stall of a cudaMalloc/cudaFree, cannot use
bsrg_mrk_cell, which allocates scratch for the interval moments.  The
allocation-free entry point keeps them in a fixed array inside the library.
This file runs last so that a failure here does not hide the other tests."""
import ctypes

import numpy as np
import pytest

from bsr_b200 import workload as W

pytestmark = pytest.mark.gpu


def _call_noalloc(basis, k, out):
    from bsr_b200._lib import call
    from bsr_b200.core import _ptr, _stream
    call("bsrg_mrk_cell_noalloc", basis.handle, k, _ptr(out), out.shape[2], _stream())
    return out


def test_noalloc_matches_mrk_cell_twice():
    """Two calls in a row through the C ABI equal bsrg_mrk_cell (same arithmetic: bit for bit)."""
    import torch

    import bsr_b200 as bsr
    cfg = W.CONFIGS["config2"]
    t, _ = W.knot_grid(cfg["ks"], cfg["ns"], cfg["rmin"], cfg["rmax"])
    basis = bsr.define_spline(t, cfg["ks"])
    out = bsr.fortran_empty((basis.ns, basis.ns, basis.ks, basis.ks))
    for k in (2, 5):
        out.fill_(float("nan"))
        _call_noalloc(basis, k, out)
        ref = bsr.mrk_cell(basis, k)
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.array_equal(a, b), k


def test_noalloc_smaller_basis_after_larger():
    """A smaller basis after a larger one: the shared array keeps the larger
    call's moments in its tail, and none of them may leak into the result."""
    import torch

    import bsr_b200 as bsr
    big = W.CONFIGS["config2"]
    t, _ = W.knot_grid(big["ks"], big["ns"], big["rmin"], big["rmax"])
    b1 = bsr.define_spline(t, big["ks"])
    o1 = bsr.fortran_empty((b1.ns, b1.ns, b1.ks, b1.ks))
    _call_noalloc(b1, 3, o1)
    small = W.CONFIGS["config1"]
    t2, _ = W.knot_grid(small["ks"], small["ns"], small["rmin"], small["rmax"])
    b2 = bsr.define_spline(t2, small["ks"])
    o2 = bsr.fortran_empty((b2.ns, b2.ns, b2.ks, b2.ks))
    for k in (3, 1):
        o2.fill_(float("nan"))
        _call_noalloc(b2, k, o2)
        ref = bsr.mrk_cell(b2, k)
        torch.cuda.synchronize()
        assert np.array_equal(o2.cpu().numpy(), ref.cpu().numpy()), k


def test_noalloc_rejects_bases_beyond_the_scratch():
    import bsr_b200 as bsr
    t, _ = W.knot_grid(10, 320, 1e-3, 60.0)          # nv = 311 > 250 for ks = 10
    basis = bsr.define_spline(t, 10)
    out = bsr.fortran_empty((basis.ns, basis.ns, 10, 10))
    with pytest.raises(bsr.BsrgError) as ei:
        _call_noalloc(basis, 0, out)
    assert "scratch" in str(ei.value)
