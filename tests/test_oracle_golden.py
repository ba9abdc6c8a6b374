"""The oracle against the reference's own known answers (src/libs/BS/TEST_BS).

int_out holds the reference's 16-digit outputs of R^k integrals by several
routes on the TEST_BS grid; int_inp1 holds exact hydrogenic rationals."""
import numpy as np
import pytest

from oracle import oracle as O


def test_gauss_matches_reference_table(golden):
    for k, tab in golden["gauss"].items():
        x, w = O.gauss(int(k))
        assert np.max(np.abs(x - np.array(tab["x"]))) < 2e-15
        assert np.max(np.abs(w - np.array(tab["w"]))) < 2e-15


def test_test_bs_grid(test_bs):
    g = test_bs["grid"]
    assert (g["ns"], g["ml"], g["me"]) == (64, 8, 49)
    assert g["t"][8] == 0.0625 and abs(g["t"][-1] - 160.48838) < 1e-5


@pytest.mark.parametrize("route", ["RK_cell", "RKd", "RKe", "RKv"])
def test_int_out_routes(test_bs, golden, route):
    B, orbs = test_bs["basis"], test_bs["orbs"]
    worst = 0.0
    for e in golden["int_out"]:
        rkb = B.mrk_cell(e["k"])
        p = [orbs[o] for o in e["orbs"]]
        got = O.rk_routes(B.ns, B.ks, rkb, *p)[route]
        ref = e["routes"][route]
        worst = max(worst, abs(got - ref) / abs(ref))
    assert worst < 1e-13, worst


def test_int_inp1_analytic_rk(test_bs, golden):
    """R^k of Z=2 hydrogenic orbitals against the exact rationals (x Z, test_bs.f90:328)."""
    B = test_bs["basis"]
    z = test_bs["knot"]["z"]
    orbs = {}
    for n in range(1, 6):
        for l in range(n):
            orbs["%d%s" % (n, "spdfg"[l])] = B.bhwf(n, l, z)
    n = 0
    for e in golden["int_inp1"]:
        if e["int"] != "R":
            continue
        rkb = B.mrk_cell(e["k"])
        p = [orbs[o] for o in e["orbs"]]
        got = O.rk_routes(B.ns, B.ks, rkb, *p)["RK_cell"]
        sa = e["ratio"] * z
        assert abs(got - sa) / abs(sa) < 1e-12, (e, got, sa)
        n += 1
    assert n >= 7


def test_orthogonality_matches_quadr_out(test_bs, golden):
    """<i|j> - delta_ij (QUADR, quadr.f90) against the 3-digit values of quadr_out,
    which the reference printed for the t.f90 orbitals (Z=2 for 1s, Z=1 otherwise)."""
    B, orbs = test_bs["basis"], test_bs["orbs"]
    for e in golden["quadr_orth"]:
        v = B.quadr(orbs[e["a"]], orbs[e["b"]], 0) - (1.0 if e["a"] == e["b"] else 0.0)
        if abs(e["err"]) > 1e-6:
            half_ulp3 = 0.5 * 10.0 ** (np.floor(np.log10(abs(e["err"]))) - 2)   # printed with 3 digits
            assert abs(v - e["err"]) <= half_ulp3 * (1 + 1e-9), (e, v)
        else:
            assert abs(v) < 1e-12, (e, v)


def test_int_inp1_analytic_nk(test_bs, golden):
    """Breit-Pauli N^k (nk_moments + mnk_cell + the nk.f90 route, fine = 1 as the TEST_BS
    harness sets it) of Z=2 hydrogenic orbitals against int_inp1's exact values x Z^3
    (test_bs.f90:326-328), including the k = -1 entries."""
    B = test_bs["basis"]
    z = test_bs["knot"]["z"]
    orbs = {}
    for n in range(1, 6):
        for l in range(n):
            orbs["%d%s" % (n, "spdfg"[l])] = B.bhwf(n, l, z)
    n = 0
    for e in golden["int_inp1"]:
        if e["int"] != "N":
            continue
        rkb = B.mnk_cell(e["k"])
        got = O.nk(B.ns, B.ks, rkb, *[orbs[o] for o in e["orbs"]])
        sa = e["ratio"] * z ** 3
        assert abs(got - sa) / abs(sa) < 1e-13, (e, got, sa)
        n += 1
    assert n == 10


def test_mnk_cell_fine_scales():
    """mnk_cell multiplies the whole table by `fine` after the cell sums (mnk_cell.f90:78)."""
    from bsr_b200 import workload as W
    cfg = W.CONFIGS["config1"]
    t, _ = W.knot_grid(cfg["ks"], cfg["ns"], cfg["rmin"], cfg["rmax"])
    B = O.Basis(cfg["ks"], t)
    a = B.mnk_cell(1, fine=1.0)
    f = 0.25 / 137.036 ** 2
    b = B.mnk_cell(1, fine=f)
    assert np.array_equal(b, a * f)
    # not symmetric under r1 <-> r2, unlike R^k
    assert np.max(np.abs(a - a.transpose(1, 0, 3, 2))) > 1e-3 * np.max(np.abs(a))


def test_int_inp1_analytic_mk(test_bs, golden):
    """Breit-Pauli M^k (mk_moments + mmk_cell + the mk.f90 route, fine = 1) against
    int_inp1's exact values x Z^3."""
    B = test_bs["basis"]
    z = test_bs["knot"]["z"]
    orbs = {"%d%s" % (n, "spdfg"[l]): B.bhwf(n, l, z) for n in range(1, 6) for l in range(n)}
    n = 0
    for e in golden["int_inp1"]:
        if e["int"] != "M":
            continue
        got = O.mk(B.ns, B.ks, B.mmk_cell(e["k"]), *[orbs[o] for o in e["orbs"]])
        sa = e["ratio"] * z ** 3
        assert abs(got - sa) / abs(sa) < 1e-13, (e, got, sa)
        n += 1
    assert n == 7


def test_int_inp1_analytic_tk(test_bs, golden):
    """Breit-Pauli T^k (tk_moments + mtk_cell + the tk.f90 route, fine = 1) against
    int_inp1 x Z^3 to 1e-12 (measured: the exact rationals within 3.4e-14, the two
    entries the file states as 16-digit decimals within 5.5e-13)."""
    B = test_bs["basis"]
    z = test_bs["knot"]["z"]
    orbs = {"%d%s" % (n, "spdfg"[l]): B.bhwf(n, l, z) for n in range(1, 6) for l in range(n)}
    n = 0
    for e in golden["int_inp1"]:
        if e["int"] != "T":
            continue
        got = O.tk(B.ns, B.ks, B.mtk_cell(e["k"]), *[orbs[o] for o in e["orbs"]])
        sa = e["ratio"] * z ** 3
        assert abs(got - sa) / abs(sa) < 1e-12, (e, got, sa)
        n += 1
    assert n == 12


def test_int_inp1_analytic_vk(test_bs, golden):
    """Breit-Pauli V^k (vk_moments + mvk_cell + the vk.f90 route, fine = 1) against
    int_inp1 x Z^3 (measured within 1.6e-15)."""
    B = test_bs["basis"]
    z = test_bs["knot"]["z"]
    orbs = {"%d%s" % (n, "spdfg"[l]): B.bhwf(n, l, z) for n in range(1, 6) for l in range(n)}
    n = 0
    for e in golden["int_inp1"]:
        if e["int"] != "V":
            continue
        got = O.vk(B.ns, B.ks, B.mvk_cell(e["k"]), *[orbs[o] for o in e["orbs"]])
        sa = e["ratio"] * z ** 3
        assert abs(got - sa) / abs(sa) < 1e-13, (e, got, sa)
        n += 1
    assert n == 13


def test_int_inp1_analytic_wk(test_bs, golden):
    """Breit-Pauli W^k (wk_moments + mwk_cell + the wk.f90 route, fine = 1) against
    int_inp1 x Z^3: nonzero values within 1e-13 (1.9e-15 measured), the four exact zeros
    within 1e-15 absolute (~1e-17 measured)."""
    B = test_bs["basis"]
    z = test_bs["knot"]["z"]
    orbs = {"%d%s" % (n, "spdfg"[l]): B.bhwf(n, l, z) for n in range(1, 6) for l in range(n)}
    n = 0
    for e in golden["int_inp1"]:
        if e["int"] != "W":
            continue
        got = O.vk(B.ns, B.ks, B.mwk_cell(e["k"]), *[orbs[o] for o in e["orbs"]])
        sa = e["ratio"] * z ** 3
        if sa == 0.0:
            assert abs(got) < 1e-15, (e, got)
        else:
            assert abs(got - sa) / abs(sa) < 1e-13, (e, got, sa)
        n += 1
    assert n == 13


def test_int_inp1_analytic_qk(test_bs, golden):
    """Breit-Pauli Q^k (qk_moments + mqk_cell + the qk.f90 route, the tk.f90 sum,
    fine = 1) against int_inp1 x Z^3: nonzero values within 1e-13 (1.6e-14 measured),
    the exact zeros within 1e-15 absolute (~1e-17 measured)."""
    B = test_bs["basis"]
    z = test_bs["knot"]["z"]
    orbs = {"%d%s" % (n, "spdfg"[l]): B.bhwf(n, l, z) for n in range(1, 6) for l in range(n)}
    n = 0
    for e in golden["int_inp1"]:
        if e["int"] != "Q":
            continue
        got = O.tk(B.ns, B.ks, B.mqk_cell(e["k"]), *[orbs[o] for o in e["orbs"]])
        sa = e["ratio"] * z ** 3
        if sa == 0.0:
            assert abs(got) < 1e-15, (e, got)
        else:
            assert abs(got - sa) / abs(sa) < 1e-13, (e, got, sa)
        n += 1
    assert n == 14


def test_mqk_cell_antisymmetric():
    """mqk_cell adds each cell term to rkb(i,j,ip,jp) and subtracts it from
    rkb(j,i,jp,ip), so the table is antisymmetric under that swap."""
    ks, ns = 5, 14
    t = np.concatenate([np.zeros(ks - 1), np.linspace(0.0, 6.0, ns - ks + 2), np.full(ks - 1, 6.0)])
    ob = O.Basis(ks, t)
    r = ob.mqk_cell(1, fine=1.0)
    assert np.max(np.abs(r + r.transpose(1, 0, 3, 2))) <= 1e-15 * np.max(np.abs(r))

