"""bsr_b200 -- B200 (sm_100a) implementation of the BSR radial, assembly and
eigensolve hot path behind the reference's routine interface.

    import bsr_b200 as bsr
    basis = bsr.define_spline(t, ks)             # define_spline
    rkb = bsr.mrk_cell(basis, k)                 # mrk_cell
    d = bsr.density(ns, ks, p1, p2, 's')         # density
    a = bsr.convol(ns, ks, d, rkb, 1, 's', 's')  # convol
    ctx = bsr.Context()
    H = bsr.assemble(ctx, basis, z, lch, ech, P, kmax, coefs)   # bsr_mat SUB1
    E = bsr.diag_hd(ctx, basis, lch, H["hcc"])                  # bsr_hd diag_hd

The compute runs in libbsrgpu.so (C ABI: include/bsr_b200.h); importing the
package does not load it, the first call does and raises if it is missing.
"""
from ._lib import LIB_PATH, BsrgError, lib  # noqa: F401
from . import workload  # noqa: F401


def __getattr__(name):
    # the torch-backed API is imported lazily so that host-only users
    # (workload generation, the C ABI symbol checks) do not need a GPU
    import importlib
    if name.startswith("__"):
        raise AttributeError(name)
    core = importlib.import_module(__name__ + ".core")
    if name == "core":
        return core
    try:
        return getattr(core, name)
    except AttributeError:
        raise AttributeError("module 'bsr_b200' has no attribute %r" % name) from None
