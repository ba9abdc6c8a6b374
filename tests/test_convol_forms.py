"""The gather form of convol used by the GPU kernels equals the reference's
scatter loops (convol.f90:2) in all 12 icase/symmetry cases.

Numpy restates the GPU's index mapping; the oracle restates convol literally.
Small random inputs (ldp = 2ks-1 so the 'n' cases have their full band)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import rel_err


def _pair(sym, ns, ks, x, xp):
    dx = xp - x
    if not (-ks < dx < ks and 0 <= x < ns and 0 <= xp < ns):
        return None
    if sym == "s":
        return (x, dx) if dx >= 0 else (xp, -dx)
    return (x, dx + ks - 1)


def _bands(sym, ns, ks, c):
    if sym == "s":
        return 0, ns - 1 - c
    return max(0, ks - 1 - c), min(ns - 1, ns - 1 + ks - 1 - c)


def gather_convol(ns, ks, d, rkb, icase, si, sj):
    a = np.zeros((ns, ns))
    if icase in (1, 2):
        so, sc = (si, sj) if icase == 1 else (sj, si)
        nco = ks if so == "s" else 2 * ks - 1
        ncc = ks if sc == "s" else 2 * ks - 1
        for op in range(nco):
            lo, hi = _bands(so, ns, ks, op)
            for o in range(lo, hi + 1):
                c = 0.0
                for cp in range(ncc):
                    clo, chi = _bands(sc, ns, ks, cp)
                    for q in range(clo, chi + 1):
                        r = rkb[o, q, op, cp] if icase == 1 else rkb[q, o, cp, op]
                        c += d[q, cp] * r
                a[o, op] = c
        return a
    for u in range(ns):
        for v in range(ns):
            c = 0.0
            for e in range(-(ks - 1), ks):
                for f in range(-(ks - 1), ks):
                    if icase == 3:
                        x, xp, yp, y = u, u + e, v, v + f
                    else:
                        xp, x, y, yp = u, u + e, v, v + f
                    m1 = _pair(si, ns, ks, x, xp)
                    m2 = _pair(sj, ns, ks, y, yp)
                    if m1 is None or m2 is None:
                        continue
                    dv = d[xp, y] if icase == 3 else d[x, yp]
                    c += rkb[m1[0], m2[0], m1[1], m2[1]] * dv
            a[u, v] = c
    return a


@pytest.mark.parametrize("icase", [1, 2, 3, 4])
@pytest.mark.parametrize("syms", ["ss", "nn", "ns", "sn"])
def test_gather_equals_scatter(icase, syms):
    rng = np.random.default_rng(7 + icase)
    ns, ks = 11, 3
    ldp = 2 * ks - 1
    rkb = np.asfortranarray(rng.standard_normal((ns, ns, ldp, ldp)))
    d = np.asfortranarray(rng.standard_normal((ns, ns)))
    ref = O.convol(ns, ks, d, rkb, icase, syms[0], syms[1])
    got = gather_convol(ns, ks, d, rkb, icase, syms[0], syms[1])
    if icase <= 2:
        so = syms[0] if icase == 1 else syms[1]
        w = ks if so == "s" else 2 * ks - 1
        ref, got = ref[:, :w], got[:, :w]
    assert rel_err(got, ref) < 1e-14


def test_convol_unknown_case():
    ns, ks = 6, 2
    with pytest.raises(ValueError):
        O.convol(ns, ks, np.zeros((ns, ns)), np.zeros((ns, ns, ks, ks)), 5, "s", "s")
