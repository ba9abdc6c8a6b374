"""The banded helpers of libs/BS on the GPU against the oracle: bav, bvmv and QUADR
bit for bit (same summation order as the reference, no FMA contraction), the
full overlap bb of initas bit for bit, and facsb's banded Cholesky factor bs
against LAPACK DPBTRF (a different summation order: 1e-13 relative)."""
import numpy as np
import pytest

from bsr_b200 import workload as W
from oracle import oracle as O
from tests.gpu_helpers import grids, to_np

pytestmark = pytest.mark.gpu


def _basis(name):
    for g in grids():
        if g[0] == name:
            return g
    raise KeyError(name)


@pytest.mark.parametrize("gname", ["test_bs", "config1", "config2"])
def test_bav_bvmv_quadr_bitwise(gname):
    import bsr_b200 as bsr
    import torch
    _, ks, t, ml, me, h = _basis(gname)
    gb = bsr.define_spline(t, ks, ml, me, h)
    ob = O.Basis(ks, t, ml, me, h)
    ns = gb.ns
    rng = np.random.default_rng(3)
    v = rng.standard_normal(ns)
    bs_ = np.asfortranarray(rng.standard_normal((ns, ks)))
    bn = np.asfortranarray(rng.standard_normal((ns, 2 * ks - 1)))
    for typ, b in (("s", bs_), ("n", bn)):
        for side in (("r",) if typ == "s" else ("r", "l")):
            got = to_np(bsr.bav(ns, ks, torch.from_numpy(b.T.copy()).T.cuda(), torch.from_numpy(v).cuda(), typ, side))
            assert np.array_equal(got, O.bav(ns, ks, b, v, typ, side)), (typ, side)
    x, y = rng.standard_normal(ns), rng.standard_normal(ns)
    for typ, b in (("s", bs_), ("a", bs_), ("g", bn)):
        got = float(to_np(bsr.bvmv(ns, ks, torch.from_numpy(b.T.copy()).T.cuda(), typ, torch.from_numpy(x).cuda(),
                                   torch.from_numpy(y).cuda()))[0])
        assert got == O.bvmv(ns, ks, b, typ, x, y), typ
    for m in (-3, -2, -1, 0, 1, 2):
        got = float(to_np(bsr.quadr(gb, torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(), m))[0])
        assert got == ob.quadr(x, y, m), m


@pytest.mark.parametrize("gname", ["test_bs", "config1", "config2"])
def test_bb_and_facsb(gname):
    import bsr_b200 as bsr
    _, ks, t, ml, me, h = _basis(gname)
    gb = bsr.define_spline(t, ks, ml, me, h)
    ns = gb.ns
    sb = to_np(gb.get("sb"))
    bb = to_np(gb.get("bb"))
    ref = np.zeros((ns, ns))
    for jc in range(ks):
        for i in range(ks - 1 - jc, ns):
            j = i + jc - ks + 1
            ref[i, j] = ref[j, i] = sb[i, jc]
    assert np.array_equal(bb, ref)
    bs = to_np(gb.get("bs"))
    rb = O.facsb(sb, ns, ks)
    assert np.max(np.abs(bs - rb)) <= 1e-13 * np.max(np.abs(rb))
