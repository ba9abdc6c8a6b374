"""Breit-Pauli N^k cell moments and tables on the GPU against the oracle: bit for bit.

nk_moments (nk_moments.f90:2) and mnk_cell (mnk_cell.f90:2) run in the
reference's summation order without fused multiply-adds, as the R^k tables do;
the N^k integrals of the TEST_BS hydrogenic orbitals computed from the GPU table
reproduce int_inp1's exact values."""
import numpy as np
import pytest

from tests.gpu_helpers import grids, to_np

pytestmark = pytest.mark.gpu

GRIDS = grids()


@pytest.fixture(scope="module", params=GRIDS, ids=[g[0] for g in GRIDS])
def pair(request):
    import bsr_b200 as bsr
    from oracle import oracle as O
    name, ks, t, ml, me, h = request.param
    return name, bsr.define_spline(t, ks, ml, me, h), O.Basis(ks, t, ml, me, h)


@pytest.mark.parametrize("k", [-1, 0, 2])
def test_nk_moments_bitwise(pair, k):
    from bsr_b200 import core
    name, gb, ob = pair
    if name == "config2" and k != 2:
        pytest.skip("one multipole suffices at ns=200")
    got = [to_np(x) for x in core.nk_moments(gb, k)]
    ref = ob.nk_moments(k)
    for g, r in zip(got, ref):
        assert np.array_equal(g, r), name


@pytest.mark.parametrize("k,fine", [(-1, 1.0), (1, 1.0), (3, 0.25 / 137.036 ** 2)])
def test_mnk_cell_bitwise(pair, k, fine):
    from bsr_b200 import core
    name, gb, ob = pair
    if name == "config2" and k != 3:
        pytest.skip("one multipole suffices at ns=200")
    got = to_np(core.mnk_cell(gb, k, fine=fine))
    ref = ob.mnk_cell(k, fine=fine)
    assert got.shape == ref.shape
    assert np.array_equal(got, ref), name


def test_mnk_cell_wide_ldp_zero(pair):
    from bsr_b200 import core
    name, gb, ob = pair
    if name != "config1":
        pytest.skip("layout check on one grid")
    ks = gb.ks
    got = to_np(core.mnk_cell(gb, 1, fine=1.0, ldp=2 * ks - 1))
    assert np.array_equal(got[:, :, :ks, :ks], ob.mnk_cell(1, fine=1.0))
    assert not np.any(got[:, :, ks:, :]) and not np.any(got[:, :, :, ks:])


def test_int_inp1_nk_on_gpu(golden, test_bs):
    """N^k of the Z=2 hydrogenic orbitals from the GPU tables against int_inp1 (x Z^3)."""
    import bsr_b200 as bsr
    from bsr_b200 import core
    from oracle import oracle as O
    B = test_bs["basis"]
    g = test_bs["grid"]
    gb = bsr.define_spline(g["t"], B.ks, g["ml"], g["me"], g["h"])
    z = test_bs["knot"]["z"]
    orbs = {"%d%s" % (n, "spdfg"[l]): B.bhwf(n, l, z) for n in range(1, 6) for l in range(n)}
    n = 0
    for e in golden["int_inp1"]:
        if e["int"] != "N":
            continue
        rkb = to_np(core.mnk_cell(gb, e["k"], fine=1.0))
        got = O.nk(B.ns, B.ks, rkb, *[orbs[o] for o in e["orbs"]])
        sa = e["ratio"] * z ** 3
        assert abs(got - sa) / abs(sa) < 1e-13, (e, got, sa)
        n += 1
    assert n == 10


def test_bad_k_rejected():
    import bsr_b200 as bsr
    from bsr_b200 import core
    from bsr_b200._lib import BsrgError
    from bsr_b200 import workload as W
    cfg = W.CONFIGS["config1"]
    t, _ = W.knot_grid(cfg["ks"], cfg["ns"], cfg["rmin"], cfg["rmax"])
    gb = bsr.define_spline(t, cfg["ks"])
    with pytest.raises(BsrgError, match="out of range"):
        core.mnk_cell(gb, -2)


@pytest.mark.parametrize("k", [-1, 1])
def test_mk_moments_and_mmk_cell_bitwise(pair, k):
    from bsr_b200 import core
    name, gb, ob = pair
    if name == "config2" and k != 1:
        pytest.skip("one multipole suffices at ns=200")
    got = [to_np(x) for x in core.mk_moments(gb, k)]
    for g, r in zip(got, ob.mk_moments(k)):
        assert np.array_equal(g, r), name
    f = 0.25 / 137.036 ** 2
    assert np.array_equal(to_np(core.mmk_cell(gb, k, fine=f)), ob.mmk_cell(k, fine=f)), name


def test_int_inp1_mk_on_gpu(golden, test_bs):
    """M^k (mk.f90 route: the rk.f90 sum halved) from the GPU tables against int_inp1 (x Z^3)."""
    import bsr_b200 as bsr
    from bsr_b200 import core
    from oracle import oracle as O
    B = test_bs["basis"]
    g = test_bs["grid"]
    gb = bsr.define_spline(g["t"], B.ks, g["ml"], g["me"], g["h"])
    z = test_bs["knot"]["z"]
    orbs = {"%d%s" % (n, "spdfg"[l]): B.bhwf(n, l, z) for n in range(1, 6) for l in range(n)}
    n = 0
    for e in golden["int_inp1"]:
        if e["int"] != "M":
            continue
        rkb = to_np(core.mmk_cell(gb, e["k"], fine=1.0))
        got = O.mk(B.ns, B.ks, rkb, *[orbs[o] for o in e["orbs"]])
        sa = e["ratio"] * z ** 3
        assert abs(got - sa) / abs(sa) < 1e-13, (e, got, sa)
        n += 1
    assert n == 7


@pytest.mark.parametrize("k", [0, 2])
def test_tk_moments_and_mtk_cell_bitwise(pair, k):
    from bsr_b200 import core
    name, gb, ob = pair
    if name == "config2" and k != 2:
        pytest.skip("one multipole suffices at ns=200")
    got = [to_np(x) for x in core.tk_moments(gb, k)]
    for g, r in zip(got, ob.tk_moments(k)):
        assert np.array_equal(g, r), name
    f = 0.25 / 137.036 ** 2
    assert np.array_equal(to_np(core.mtk_cell(gb, k, fine=f)), ob.mtk_cell(k, fine=f)), name


def test_int_inp1_tk_on_gpu(golden, test_bs):
    """T^k (tk.f90 route) from the GPU tables against int_inp1 (x Z^3) to 1e-12."""
    import bsr_b200 as bsr
    from bsr_b200 import core
    from oracle import oracle as O
    B = test_bs["basis"]
    g = test_bs["grid"]
    gb = bsr.define_spline(g["t"], B.ks, g["ml"], g["me"], g["h"])
    z = test_bs["knot"]["z"]
    orbs = {"%d%s" % (n, "spdfg"[l]): B.bhwf(n, l, z) for n in range(1, 6) for l in range(n)}
    n = 0
    for e in golden["int_inp1"]:
        if e["int"] != "T":
            continue
        rkb = to_np(core.mtk_cell(gb, e["k"], fine=1.0))
        got = O.tk(B.ns, B.ks, rkb, *[orbs[o] for o in e["orbs"]])
        sa = e["ratio"] * z ** 3
        assert abs(got - sa) / abs(sa) < 1e-12, (e, got, sa)
        n += 1
    assert n == 12


@pytest.mark.parametrize("k", [0, 1])
def test_vk_moments_and_mvk_cell_bitwise(pair, k):
    from bsr_b200 import core
    name, gb, ob = pair
    if name == "config2" and k != 1:
        pytest.skip("one multipole suffices at ns=200")
    got = [to_np(x) for x in core.vk_moments(gb, k)]
    for g, r in zip(got, ob.vk_moments(k)):
        assert np.array_equal(g, r), name
    f = 0.25 / 137.036 ** 2
    assert np.array_equal(to_np(core.mvk_cell(gb, k, fine=f)), ob.mvk_cell(k, fine=f)), name


def test_int_inp1_vk_on_gpu(golden, test_bs):
    """V^k (vk.f90 route) from the GPU tables against int_inp1 (x Z^3)."""
    import bsr_b200 as bsr
    from bsr_b200 import core
    from oracle import oracle as O
    B = test_bs["basis"]
    g = test_bs["grid"]
    gb = bsr.define_spline(g["t"], B.ks, g["ml"], g["me"], g["h"])
    z = test_bs["knot"]["z"]
    orbs = {"%d%s" % (n, "spdfg"[l]): B.bhwf(n, l, z) for n in range(1, 6) for l in range(n)}
    n = 0
    for e in golden["int_inp1"]:
        if e["int"] != "V":
            continue
        rkb = to_np(core.mvk_cell(gb, e["k"], fine=1.0))
        got = O.vk(B.ns, B.ks, rkb, *[orbs[o] for o in e["orbs"]])
        sa = e["ratio"] * z ** 3
        assert abs(got - sa) / abs(sa) < 1e-13, (e, got, sa)
        n += 1
    assert n == 13


@pytest.mark.parametrize("k", [0, 1])
def test_wk_moments_and_mwk_cell_bitwise(pair, k):
    from bsr_b200 import core
    name, gb, ob = pair
    if name == "config2" and k != 1:
        pytest.skip("one multipole suffices at ns=200")
    got = [to_np(x) for x in core.wk_moments(gb, k)]
    for g, r in zip(got, ob.wk_moments(k)):
        assert np.array_equal(g, r), name
    f = 0.25 / 137.036 ** 2
    assert np.array_equal(to_np(core.mwk_cell(gb, k, fine=f)), ob.mwk_cell(k, fine=f)), name


def test_int_inp1_wk_on_gpu(golden, test_bs):
    """W^k (wk.f90 route, the vk.f90 sum) from the GPU tables against int_inp1 (x Z^3);
    the entries whose exact value is zero to 1e-15 absolute."""
    import bsr_b200 as bsr
    from bsr_b200 import core
    from oracle import oracle as O
    B = test_bs["basis"]
    g = test_bs["grid"]
    gb = bsr.define_spline(g["t"], B.ks, g["ml"], g["me"], g["h"])
    z = test_bs["knot"]["z"]
    orbs = {"%d%s" % (n, "spdfg"[l]): B.bhwf(n, l, z) for n in range(1, 6) for l in range(n)}
    n = 0
    for e in golden["int_inp1"]:
        if e["int"] != "W":
            continue
        rkb = to_np(core.mwk_cell(gb, e["k"], fine=1.0))
        got = O.vk(B.ns, B.ks, rkb, *[orbs[o] for o in e["orbs"]])
        sa = e["ratio"] * z ** 3
        if sa == 0.0:
            assert abs(got) < 1e-15, (e, got)
        else:
            assert abs(got - sa) / abs(sa) < 1e-13, (e, got, sa)
        n += 1
    assert n == 13


@pytest.mark.parametrize("k", [0, 1, 2])
def test_qk_moments_and_mqk_cell_bitwise(pair, k):
    """Q^k: the GPU moments and the expanded table equal the oracle's bit for bit; the
    expansion replays the reference's interleaved add/subtract order per element."""
    from bsr_b200 import core
    name, gb, ob = pair
    if name == "config2" and k != 1:
        pytest.skip("one multipole suffices at ns=200")
    got = [to_np(x) for x in core.qk_moments(gb, k)]
    for g, r in zip(got, ob.qk_moments(k)):
        assert np.array_equal(g, r), name
    f = 0.25 / 137.036 ** 2
    assert np.array_equal(to_np(core.mqk_cell(gb, k, fine=f)), ob.mqk_cell(k, fine=f)), name


def test_int_inp1_qk_on_gpu(golden, test_bs):
    """Q^k (qk.f90 route, the tk.f90 sum) from the GPU tables against int_inp1 (x Z^3);
    the entries whose exact value is zero to 1e-15 absolute."""
    import bsr_b200 as bsr
    from bsr_b200 import core
    from oracle import oracle as O
    B = test_bs["basis"]
    g = test_bs["grid"]
    gb = bsr.define_spline(g["t"], B.ks, g["ml"], g["me"], g["h"])
    z = test_bs["knot"]["z"]
    orbs = {"%d%s" % (n, "spdfg"[l]): B.bhwf(n, l, z) for n in range(1, 6) for l in range(n)}
    n = 0
    for e in golden["int_inp1"]:
        if e["int"] != "Q":
            continue
        rkb = to_np(core.mqk_cell(gb, e["k"], fine=1.0))
        got = O.tk(B.ns, B.ks, rkb, *[orbs[o] for o in e["orbs"]])
        sa = e["ratio"] * z ** 3
        if sa == 0.0:
            assert abs(got) < 1e-15, (e, got)
        else:
            assert abs(got - sa) / abs(sa) < 1e-13, (e, got, sa)
        n += 1
    assert n == 14

