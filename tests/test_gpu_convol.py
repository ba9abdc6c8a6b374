"""GPU density / convol / SUM_AmB against the oracle, and the reference's
int_out R^k values recomputed entirely on the GPU."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import rel_err
from tests.gpu_helpers import to_np

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("typ", ["s", "n", "x"])
def test_density_bitwise(typ):
    import bsr_b200 as bsr
    rng = np.random.default_rng(3)
    ns, ks = 37, 6
    p1, p2 = rng.standard_normal(ns), rng.standard_normal(ns)
    got = to_np(bsr.density(ns, ks, p1, p2, typ))
    ref = O.density(ns, ks, p1, p2, typ)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("icase", [1, 2, 3, 4])
@pytest.mark.parametrize("syms", ["ss", "nn", "ns", "sn"])
def test_convol_cases(icase, syms):
    import bsr_b200 as bsr
    rng = np.random.default_rng(11 * icase + len(syms))
    ns, ks = 29, 5
    ldp = 2 * ks - 1
    rkb = np.asfortranarray(rng.standard_normal((ns, ns, ldp, ldp)))
    d = np.asfortranarray(rng.standard_normal((ns, ns)))
    ref = O.convol(ns, ks, d, rkb, icase, syms[0], syms[1])
    got = to_np(bsr.convol(ns, ks, d, rkb, icase, syms[0], syms[1]))
    if icase <= 2:
        ref = ref[:, : got.shape[1]]
        # band results keep the reference's summation order: bit for bit
        assert np.array_equal(got, ref)
    else:
        assert rel_err(got, ref) < 1e-13


def test_convol_unknown_case_raises():
    import bsr_b200 as bsr
    ns, ks = 8, 3
    with pytest.raises(bsr.BsrgError) as ei:
        bsr.convol(ns, ks, np.zeros((ns, ns)), np.zeros((ns, ns, ks, ks)), 5, "s", "s")
    assert "CONVOL" in str(ei.value)


@pytest.mark.parametrize("sym", ["s", "l", "n", "x"])
def test_sum_amb_bitwise(sym):
    import bsr_b200 as bsr
    rng = np.random.default_rng(5)
    ns, ks = 23, 4
    a = np.asfortranarray(rng.standard_normal((ns, ns)))
    b = np.asfortranarray(rng.standard_normal((ns, ns)))
    got = float(bsr.sum_amb(ns, ks, a, b, sym).cpu()[0])
    assert got == O.sum_amb(ns, ks, a, b, sym)


def _gpu_routes(ns, ks, rkb, p):
    """RK_cell (rk.f90) and RKd/RKe (test_bs.f90 rkd/rke) from GPU density/convol/SUM_AmB."""
    import bsr_b200 as bsr
    pi1, pj1, pi2, pj2 = p
    # RK_cell: sum a(i,ip) * sum b(j,jp) rkb(j,i,jp,ip)  == SUM_AmB(convol(b, icase 2), a)
    a = bsr.density(ns, ks, pi1, pi2, "s")
    b = bsr.density(ns, ks, pj1, pj2, "s")
    x = bsr.convol(ns, ks, b, rkb, 2, "s", "s")
    rk_cell = float(bsr.sum_amb(ns, ks, x, a, "s").cpu()[0])
    # RKd
    x2 = bsr.convol(ns, ks, bsr.density(ns, ks, pi1, pi2, "s"), rkb, 2, "s", "s")
    r = float(bsr.sum_amb(ns, ks, x2, bsr.density(ns, ks, pj1, pj2, "s"), "s").cpu()[0])
    x1 = bsr.convol(ns, ks, bsr.density(ns, ks, pj1, pj2, "s"), rkb, 1, "s", "s")
    r += float(bsr.sum_amb(ns, ks, x1, bsr.density(ns, ks, pi1, pi2, "s"), "s").cpu()[0])
    rkd = r / 2
    # RKe
    x3 = bsr.convol(ns, ks, bsr.density(ns, ks, pi2, pj1, "x"), rkb, 3, "s", "s")
    r = float(bsr.sum_amb(ns, ks, x3, bsr.density(ns, ks, pi1, pj2, "x"), "x").cpu()[0])
    x4 = bsr.convol(ns, ks, bsr.density(ns, ks, pi1, pj2, "x"), rkb, 4, "s", "s")
    r += float(bsr.sum_amb(ns, ks, x4, bsr.density(ns, ks, pi2, pj1, "x"), "x").cpu()[0])
    rke = r / 2
    return {"RK_cell": rk_cell, "RKd": rkd, "RKe": rke}


def test_int_out_on_gpu(test_bs, golden):
    """The reference's own int_out R^k values (TEST_BS), every stage on the GPU."""
    import bsr_b200 as bsr
    g = test_bs["grid"]
    gb = bsr.define_spline(g["t"], g["ks"], g["ml"], g["me"], g["h"])
    ns, ks = gb.ns, gb.ks
    worst = {}
    for e in golden["int_out"]:
        rkb = bsr.mrk_cell(gb, e["k"])
        p = [test_bs["orbs"][o] for o in e["orbs"]]
        got = _gpu_routes(ns, ks, rkb, p)
        for route, v in got.items():
            ref = e["routes"][route]
            worst[route] = max(worst.get(route, 0.0), abs(v - ref) / abs(ref))
    assert all(w < 1e-13 for w in worst.values()), worst
