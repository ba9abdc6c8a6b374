"""ctypes front end of the CPU oracle (oracle/liboracle.so) plus the diag_hd restatement.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference leg as the checker.  The product
(bsr_b200/) never imports this module.

The C part restates the reference's B-spline radial library (src/libs/BS) and
the bsr_mat channel-block assembly (src/bsr/BSR_MAT3); the diag_hd part below
restates src/bsr/BSR_HD3/diag_hd.f90 with scipy's LAPACK (DSYGV, DSYEV) as the
stand-in for the system LAPACK the reference links.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_gauss.argtypes = [ctypes.c_int, _D, _D]
        L.orc_mkgrid0.argtypes = [ctypes.c_int] + [ctypes.c_double] * 4 + [_D, ctypes.c_int, _I, _I, _I, _D]
        L.orc_mkgrid1.argtypes = L.orc_mkgrid0.argtypes
        L.orc_basis_new.restype = ctypes.c_void_p
        L.orc_basis_new.argtypes = [ctypes.c_int, ctypes.c_int, _D, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.orc_basis_free.argtypes = [ctypes.c_void_p]
        L.orc_basis_get.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
        L.orc_mrm.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
        L.orc_bhwf.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, _D]
        L.orc_moments.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, ctypes.c_char, ctypes.c_char]
        L.orc_rk_moments.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, _D]
        L.orc_mrk_cell.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, ctypes.c_int]
        L.orc_density.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, ctypes.c_char]
        L.orc_convol.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_char, ctypes.c_char]
        L.orc_sum_amb.restype = ctypes.c_double
        L.orc_sum_amb.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, ctypes.c_char]
        L.orc_bav.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, ctypes.c_char, ctypes.c_char]
        L.orc_bvmv.restype = ctypes.c_double
        L.orc_bvmv.argtypes = [ctypes.c_int, ctypes.c_int, _D, ctypes.c_char, _D, _D]
        L.orc_quadr.restype = ctypes.c_double
        L.orc_quadr.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_int]
        for f in ("orc_rk", "orc_rkd", "orc_rke", "orc_rkv"):
            getattr(L, f).restype = ctypes.c_double
            getattr(L, f).argtypes = [ctypes.c_int, ctypes.c_int, _D, ctypes.c_int, _D, _D, _D, _D]
        L.orc_hl_full.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _D]
        L.orc_assemble.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, _I, _D,
                                   ctypes.c_int, _D, ctypes.c_int, _D,
                                   ctypes.c_int, _I, _I, _I, _I, _I, _I, _D, _D, _D, _D]
        L.orc_nk_moments.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, _D]
        L.orc_mnk_cell.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _D, ctypes.c_int]
        L.orc_mk_moments.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, _D]
        L.orc_mmk_cell.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _D, ctypes.c_int]
        L.orc_tk_moments.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, _D]
        L.orc_mtk_cell.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _D, ctypes.c_int]
        L.orc_tk.restype = ctypes.c_double
        L.orc_tk.argtypes = [ctypes.c_int, ctypes.c_int, _D, ctypes.c_int, _D, _D, _D, _D]
        L.orc_vk_moments.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, _D, _D, _D]
        L.orc_mvk_cell.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _D, ctypes.c_int]
        L.orc_wk_moments.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, _D, _D, _D]
        L.orc_mwk_cell.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _D, ctypes.c_int]
        L.orc_qk_moments.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, _D, _D, _D]
        L.orc_mqk_cell.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _D, ctypes.c_int]
        L.orc_vk.restype = ctypes.c_double
        L.orc_vk.argtypes = [ctypes.c_int, ctypes.c_int, _D, ctypes.c_int, _D, _D, _D, _D]
        L.orc_nk.restype = ctypes.c_double
        L.orc_nk.argtypes = [ctypes.c_int, ctypes.c_int, _D, ctypes.c_int, _D, _D, _D, _D]
        L.orc_bs_orth.argtypes = [ctypes.c_int, ctypes.c_int, _D, ctypes.c_int, _D, _I, _I, _D]
        L.orc_rsol.argtypes = [ctypes.c_int, ctypes.c_int, _I, _D, ctypes.c_int, _D, _D, _D]
        L.orc_channel_weights.argtypes = [ctypes.c_int, _I, ctypes.c_int, _D, _D, _I, _I]
        _LIB = L
    return _LIB


def build():
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _p(a):
    return a.ctypes.data_as(_D)


def _pi(a):
    return a.ctypes.data_as(_I)


def gauss(k):
    x = np.zeros(k)
    w = np.zeros(k)
    lib().orc_gauss(k, _p(x), _p(w))
    return x, w


def mkgrid(grid_type, ks, z, h, hmax, rmax):
    """define_grid (define_grid.f90:2): returns dict(t, ns, ml, me, h)."""
    cap = int((rmax * z / h + 1 + ks) * 2) + 4 * ks + 64
    t = np.zeros(cap)
    ns = ctypes.c_int()
    ml = ctypes.c_int()
    me = ctypes.c_int()
    hh = ctypes.c_double()
    f = lib().orc_mkgrid0 if grid_type == 0 else lib().orc_mkgrid1
    rc = f(ks, z, h, hmax, rmax, _p(t), cap, ctypes.byref(ns), ctypes.byref(ml), ctypes.byref(me),
           ctypes.byref(hh))
    if rc != 0:
        raise RuntimeError("mkgrid failed")
    n = ns.value
    return {"t": t[: n + ks].copy(), "ns": n, "ml": ml.value, "me": me.value, "h": hh.value, "ks": ks}


class Basis:
    """define_spline (define_spline.f90:15) state on the CPU."""

    NAMES = {"gr": 0, "grm": 1, "grw": 2, "bsp": 3, "bsq": 4, "bspd": 5, "sb": 6, "r1": 7,
             "rm1": 8, "rm2": 9, "rm3": 10, "db1": 11, "db2": 12, "gx": 13, "gw": 14}

    def __init__(self, ks, t, ml=0, me=0, h=0.0):
        t = np.ascontiguousarray(t, dtype=np.float64)
        self.ks = ks
        self.ns = len(t) - ks
        self.nv = self.ns - ks + 1
        self.ml, self.me, self.h = ml, me, h
        self.t = t
        self._h = lib().orc_basis_new(ks, self.ns, _p(t), ml, me, h)
        if not self._h:
            raise ValueError("bad basis")

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.orc_basis_free(self._h)
            self._h = None

    def get(self, name):
        ks, ns, nv = self.ks, self.ns, self.nv
        shapes = {"gr": (ks, nv), "grm": (ks, nv), "grw": (ks, nv), "bsp": (ks, ks, nv + 1),
                  "bsq": (ks, ks, nv + 1), "bspd": (2, ks, ks, nv + 1), "gx": (ks,), "gw": (ks,)}
        shp = shapes.get(name, (ks, ns))
        out = np.zeros(shp)
        lib().orc_basis_get(self._h, self.NAMES[name], _p(out))
        return out  # C-order view of the Fortran column-major array: reversed index order

    def band(self, name):
        """(ns, ks) Fortran band matrix as a numpy array indexed [i, jcol]."""
        return self.get(name).T.copy()

    def mrm(self, mm):
        out = np.zeros((self.ks, self.ns))
        lib().orc_mrm(self._h, mm, _p(out))
        return out.T.copy()

    def bhwf(self, n, l, z):
        c = np.zeros(self.ns)
        rc = lib().orc_bhwf(self._h, n, l, z, _p(c))
        if rc != 0:
            raise RuntimeError("bhwf: Cholesky failed")
        return c

    def rk_moments(self, k):
        ik = self.ks * (self.ks + 1) // 2
        rkd1 = np.zeros((self.nv, ik))
        rkd2 = np.zeros((self.nv, ik))
        rkd = np.zeros((self.nv, ik, ik))
        lib().orc_rk_moments(self._h, k, _p(rkd1), _p(rkd2), _p(rkd))
        # Fortran (ik,nv) and (ik,ik,nv) column-major -> return [iv, ii] and [iv, jj, ii]
        return rkd1, rkd2, rkd

    def mrk_cell(self, k, ldp=None):
        """rkb (ns,ns,ldp,ldp) Fortran order, returned as a flat Fortran-ordered array."""
        ldp = ldp or self.ks
        rkb = np.zeros(self.ns * self.ns * ldp * ldp)
        lib().orc_mrk_cell(self._h, k, _p(rkb), ldp)
        return rkb.reshape((self.ns, self.ns, ldp, ldp), order="F")

    def nk_moments(self, k):
        """nk_moments (nk_moments.f90:2): rkd1 (ik,nv) power k, rkd2 power -(k+3), rkd (ik,ik,nv)."""
        ik = self.ks * (self.ks + 1) // 2
        rkd1 = np.zeros(ik * self.nv)
        rkd2 = np.zeros(ik * self.nv)
        rkd = np.zeros(ik * ik * self.nv)
        lib().orc_nk_moments(self._h, k, _p(rkd1), _p(rkd2), _p(rkd))
        return (rkd1.reshape((ik, self.nv), order="F"), rkd2.reshape((ik, self.nv), order="F"),
                rkd.reshape((ik, ik, self.nv), order="F"))

    def mk_moments(self, k):
        """mk_moments (mk_moments.f90:2): as nk_moments with symmetrised diagonal cells."""
        ik = self.ks * (self.ks + 1) // 2
        rkd1 = np.zeros(ik * self.nv)
        rkd2 = np.zeros(ik * self.nv)
        rkd = np.zeros(ik * ik * self.nv)
        lib().orc_mk_moments(self._h, k, _p(rkd1), _p(rkd2), _p(rkd))
        return (rkd1.reshape((ik, self.nv), order="F"), rkd2.reshape((ik, self.nv), order="F"),
                rkd.reshape((ik, ik, self.nv), order="F"))

    def mmk_cell(self, k, fine=1.0, ldp=None):
        """mmk_cell (mmk_cell.f90:2): M^k table rkb (ns,ns,ldp,ldp), Fortran order, times fine."""
        ldp = ldp or self.ks
        rkb = np.zeros(self.ns * self.ns * ldp * ldp)
        lib().orc_mmk_cell(self._h, k, float(fine), _p(rkb), ldp)
        return rkb.reshape((self.ns, self.ns, ldp, ldp), order="F")

    def tk_moments(self, k):
        """tk_moments (tk_moments.f90:2): rkd1, rkd2 (ks*ks, nv) 'n','d' moments, rkd (ks*ks, ks*ks, nv)."""
        jk = self.ks * self.ks
        rkd1 = np.zeros(jk * self.nv)
        rkd2 = np.zeros(jk * self.nv)
        rkd = np.zeros(jk * jk * self.nv)
        lib().orc_tk_moments(self._h, k, _p(rkd1), _p(rkd2), _p(rkd))
        return (rkd1.reshape((jk, self.nv), order="F"), rkd2.reshape((jk, self.nv), order="F"),
                rkd.reshape((jk, jk, self.nv), order="F"))

    def mtk_cell(self, k, fine=1.0, ldp=None):
        """mtk_cell (mtk_cell.f90:2): T^k table (ns,ns,ldp,ldp), ldp >= 2ks-1, times fine/(2k+1)."""
        ldp = ldp or 2 * self.ks - 1
        rkb = np.zeros(self.ns * self.ns * ldp * ldp)
        lib().orc_mtk_cell(self._h, k, float(fine), _p(rkb), ldp)
        return rkb.reshape((self.ns, self.ns, ldp, ldp), order="F")

    def vk_moments(self, k):
        """vk_moments (vk_moments.f90:2): rkd1, rkd2 (ik, nv), rkd3, rkd4 (ks*ks, nv), rkd (ks*ks, ik, nv)."""
        ik, jk, nv = self.ks * (self.ks + 1) // 2, self.ks * self.ks, self.nv
        r1, r2, r3, r4 = np.zeros(ik * nv), np.zeros(ik * nv), np.zeros(jk * nv), np.zeros(jk * nv)
        rd = np.zeros(jk * ik * nv)
        lib().orc_vk_moments(self._h, k, _p(r1), _p(r2), _p(r3), _p(r4), _p(rd))
        return (r1.reshape((ik, nv), order="F"), r2.reshape((ik, nv), order="F"), r3.reshape((jk, nv), order="F"),
                r4.reshape((jk, nv), order="F"), rd.reshape((jk, ik, nv), order="F"))

    def wk_moments(self, k):
        """wk_moments (wk_moments.f90:2): the V^k layouts with W^k's combined moments and operators."""
        ik, jk, nv = self.ks * (self.ks + 1) // 2, self.ks * self.ks, self.nv
        r1, r2, r3, r4 = np.zeros(ik * nv), np.zeros(ik * nv), np.zeros(jk * nv), np.zeros(jk * nv)
        rd = np.zeros(jk * ik * nv)
        lib().orc_wk_moments(self._h, k, _p(r1), _p(r2), _p(r3), _p(r4), _p(rd))
        return (r1.reshape((ik, nv), order="F"), r2.reshape((ik, nv), order="F"), r3.reshape((jk, nv), order="F"),
                r4.reshape((jk, nv), order="F"), rd.reshape((jk, ik, nv), order="F"))

    def mwk_cell(self, k, fine=1.0, ldp=None):
        """mwk_cell (mwk_cell.f90:2): W^k table (ns,ns,ldp,ldp), ldp >= 2ks-1, times fine."""
        ldp = ldp or 2 * self.ks - 1
        rkb = np.zeros(self.ns * self.ns * ldp * ldp)
        lib().orc_mwk_cell(self._h, k, float(fine), _p(rkb), ldp)
        return rkb.reshape((self.ns, self.ns, ldp, ldp), order="F")

    def qk_moments(self, k):
        """qk_moments (qk_moments.f90:2): rkd1..rkd4 (ks*ks, nv), rkd (ks*ks, ks*ks, nv)."""
        jk, nv = self.ks * self.ks, self.nv
        r = [np.zeros(jk * nv) for _ in range(4)]
        rd = np.zeros(jk * jk * nv)
        lib().orc_qk_moments(self._h, k, *[_p(x) for x in r], _p(rd))
        return tuple(x.reshape((jk, nv), order="F") for x in r) + (rd.reshape((jk, jk, nv), order="F"),)

    def mqk_cell(self, k, fine=1.0, ldp=None):
        """mqk_cell (mqk_cell.f90:2): Q^k table (ns,ns,ldp,ldp), ldp >= 2ks-1, times fine."""
        ldp = ldp or 2 * self.ks - 1
        rkb = np.zeros(self.ns * self.ns * ldp * ldp)
        lib().orc_mqk_cell(self._h, k, float(fine), _p(rkb), ldp)
        return rkb.reshape((self.ns, self.ns, ldp, ldp), order="F")

    def mvk_cell(self, k, fine=1.0, ldp=None):
        """mvk_cell (mvk_cell.f90:2): V^k table (ns,ns,ldp,ldp), ldp >= 2ks-1, times fine."""
        ldp = ldp or 2 * self.ks - 1
        rkb = np.zeros(self.ns * self.ns * ldp * ldp)
        lib().orc_mvk_cell(self._h, k, float(fine), _p(rkb), ldp)
        return rkb.reshape((self.ns, self.ns, ldp, ldp), order="F")

    def mnk_cell(self, k, fine=1.0, ldp=None):
        """mnk_cell (mnk_cell.f90:2): N^k table rkb (ns,ns,ldp,ldp), Fortran order, times fine."""
        ldp = ldp or self.ks
        rkb = np.zeros(self.ns * self.ns * ldp * ldp)
        lib().orc_mnk_cell(self._h, k, float(fine), _p(rkb), ldp)
        return rkb.reshape((self.ns, self.ns, ldp, ldp), order="F")

    def quadr(self, p1, p2, m):
        p1 = np.ascontiguousarray(p1, dtype=np.float64)
        p2 = np.ascontiguousarray(p2, dtype=np.float64)
        return lib().orc_quadr(self._h, _p(p1), _p(p2), m)

    def hl_full(self, l, z):
        out = np.zeros((self.ns, self.ns))
        lib().orc_hl_full(self._h, l, z, _p(out))
        return out.T.copy()


def density(ns, ks, p1, p2, typ):
    cols = {"s": ks, "n": 2 * ks - 1}.get(typ, ns)
    d = np.zeros(ns * max(cols, ns))
    lib().orc_density(ns, ks, _p(d), _p(np.ascontiguousarray(p1, dtype=np.float64)),
                      _p(np.ascontiguousarray(p2, dtype=np.float64)), typ.encode())
    return d.reshape((ns, -1), order="F")[:, :cols].copy(order="F")


def convol(ns, ks, d, rkb, icase, sym_i, sym_j):
    """convol.f90:2.  d (ns, *) Fortran-ordered; rkb (ns,ns,ldp,ldp) Fortran-ordered."""
    ldp = rkb.shape[2]
    dd = np.zeros((ns, ns), order="F")
    dd[:, : d.shape[1]] = d
    a = np.zeros((ns, ns), order="F")
    rk = np.asfortranarray(rkb)
    rc = lib().orc_convol(ns, ks, a.ctypes.data_as(_D), dd.ctypes.data_as(_D), rk.ctypes.data_as(_D),
                          ldp, icase, sym_i.encode(), sym_j.encode())
    if rc != 0:
        raise ValueError("convol: unknown case")
    return a


def bav(ns, ks, b, v, typ, side="r"):
    """bav.f90:2 (y = B v or v B for a band matrix)."""
    b = np.asfortranarray(b, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    y = np.zeros(ns)
    lib().orc_bav(ns, ks, _p(b), _p(v), _p(y), typ.encode(), side.encode())
    return y


def bvmv(n, k, ar, typ, x, y):
    """bvmv.f90:2 (<x, A y> for a band array)."""
    ar = np.asfortranarray(ar, dtype=np.float64)
    return lib().orc_bvmv(n, k, _p(ar), typ.encode(), _p(np.ascontiguousarray(x, dtype=np.float64)),
                          _p(np.ascontiguousarray(y, dtype=np.float64)))


def facsb(sb, ns, ks):
    """facsb.f90:2-36: bs = sb^T (upper band storage (ks, ns)) with the r = 0 boundary
    condition, factorised by LAPACK DPBTRF('U') (scipy's, standing in for the reference's)."""
    from scipy.linalg import lapack
    bs = np.asfortranarray(np.asarray(sb).T.copy())
    for m in range(ks - 1):
        bs[m, ks - 1 - m] = 0.0
    bs[ks - 1, 0] = 1.0
    c, info = lapack.dpbtrf(bs, lower=0)
    if info != 0:
        raise RuntimeError("facsb: dpbtrf (LAPACK) failed")
    return np.asfortranarray(c)


def sum_amb(ns, ks, a, b, sym):
    cols = ns
    aa = np.zeros((ns, cols), order="F")
    bb = np.zeros((ns, cols), order="F")
    aa[:, : a.shape[1]] = a
    bb[:, : b.shape[1]] = b
    return lib().orc_sum_amb(ns, ks, aa.ctypes.data_as(_D), bb.ctypes.data_as(_D), sym.encode())


def rk_routes(ns, ks, rkb, pi1, pj1, pi2, pj2):
    """R^k(i1,j1;i2,j2) by the table (rk.f90), direct (rkd), exchange (rke) and vector (rkv) routes."""
    rk = np.asfortranarray(rkb)
    ldp = rkb.shape[2]
    args = [np.ascontiguousarray(x, dtype=np.float64) for x in (pi1, pj1, pi2, pj2)]
    L = lib()
    out = {}
    for name, f in (("RK_cell", L.orc_rk), ("RKd", L.orc_rkd), ("RKe", L.orc_rke), ("RKv", L.orc_rkv)):
        out[name] = f(ns, ks, rk.ctypes.data_as(_D), ldp, *[_p(a) for a in args])
    return out


def assemble(basis, z, lch, ech, P, kmax, rkb_all, coefs, want_s=True, want_acf=True):
    """bsr_mat SUB1 for one partial wave (channel-channel part).

    rkb_all: (ns,ns,ks,ks,kmax+1) Fortran-ordered.  coefs: dict of int arrays
    k, type, ich, jch, a, b and float array c, sorted by (k, type, ich, jch).
    Returns hcc (nblk, ns, ns) with hcc[ij] the Fortran (ns,ns) block as a
    C-order array indexed [col, row] -> we transpose to [row, col].
    """
    ns, ks = basis.ns, basis.ks
    nch = len(lch)
    nblk = nch * (nch + 1) // 2
    hcc = np.zeros(nblk * ns * ns)
    scc = np.zeros(nblk * ns * ns) if want_s else None
    acf = np.zeros(nch * nch * (kmax + 1)) if want_acf else None
    lch_a = np.ascontiguousarray(lch, dtype=np.int32)
    ech_a = np.ascontiguousarray(ech, dtype=np.float64)
    Pf = np.asfortranarray(P, dtype=np.float64)
    rk = np.asfortranarray(rkb_all)
    c = {kk: np.ascontiguousarray(coefs[kk], dtype=np.int32) for kk in ("k", "type", "ich", "jch", "a", "b")}
    cv = np.ascontiguousarray(coefs["c"], dtype=np.float64)
    rc = lib().orc_assemble(basis._h, z, nch, _pi(lch_a), _p(ech_a), P.shape[1], Pf.ctypes.data_as(_D),
                            kmax, rk.ctypes.data_as(_D), len(cv), _pi(c["k"]), _pi(c["type"]),
                            _pi(c["ich"]), _pi(c["jch"]), _pi(c["a"]), _pi(c["b"]), _p(cv), _p(hcc),
                            _p(scc) if want_s else None, _p(acf) if want_acf else None)
    if rc != 0:
        raise ValueError("assemble: coefficient out of range")
    out = {"hcc": hcc.reshape(nblk, ns, ns).transpose(0, 2, 1).copy()}
    if want_s:
        out["scc"] = scc.reshape(nblk, ns, ns).transpose(0, 2, 1).copy()
    if want_acf:
        out["acf"] = acf.reshape(kmax + 1, nch, nch).transpose(0, 2, 1).copy()
    return out


# ---------------------------------------------------------------------------
# diag_hd restatement (src/bsr/BSR_HD3/diag_hd.f90:2-340) with scipy LAPACK
# ---------------------------------------------------------------------------
RR_HW = 8   # half-width of the Rayleigh-Ritz window of rayleigh_refine


def jacobi_eigvals(M, sweeps=10):
    """Eigenvalues of the small symmetric M by cyclic Jacobi rotations (each zeroes one
    off-diagonal pair; tan of its angle = the smaller root of t^2 + 2 theta t - 1 = 0,
    theta = (a_qq - a_pp) / (2 a_pq)), unsorted.  Rotations keep small eigenvalues of a
    graded matrix to relative accuracy, where a tridiagonalising solver is off by
    ~eps ||M||.  The sequence of rotations is the library's (refine.cu)."""
    A = np.array(M, dtype=np.float64)
    w = A.shape[0]
    for _ in range(sweeps):
        rotated = False
        for p in range(w - 1):
            for q in range(p + 1, w):
                apq, app, aqq = A[p, q], A[p, p], A[q, q]
                if not (abs(apq) > 1e-19 * (abs(app) + abs(aqq))) or abs(apq) < 1e-300:
                    continue
                rotated = True
                th = (aqq - app) / (2.0 * apq)
                t = 0.5 / th if abs(th) > 1e150 else np.copysign(1.0, th) / (abs(th) + np.sqrt(1.0 + th * th))
                c = 1.0 / np.sqrt(1.0 + t * t)
                s = t * c
                k = np.array([i for i in range(w) if i != p and i != q], dtype=int)
                akp, akq = A[k, p].copy(), A[k, q].copy()
                A[k, p] = A[p, k] = c * akp - s * akq
                A[k, q] = A[q, k] = s * akp + c * akq
                A[p, p] = app - t * apq
                A[q, q] = aqq + t * apq
                A[p, q] = A[q, p] = 0.0
        if not rotated:
            break
    return np.diag(A).copy()


def rayleigh_refine(A, ev, V, dtype=np.longdouble, window=RR_HW):
    """Refined eigenvalues of the eigenpairs (ev, V) of the symmetric A, evaluated in `dtype`
    (long double: ~1e-19 relative rounding).  The Rayleigh quotient lambda + v^T r / v^T v
    (r = A v - lambda v) leaves an error ~||r||^2 / gap, which close pairs feel; so, as the
    library does (refine.cu), each lambda_j becomes the Rayleigh-Ritz value in j's place of
    the window of pairs [j - window, j + window] (cut to the pairs given):
    M(k, l) = (v_k^T r_l + lambda_l v_k^T v_l) / (|v_k| |v_l|), symmetrised, its eigenvalues
    by jacobi_eigvals.  window=0 gives the plain quotients.
    Returns (refined eigenvalues in the order of ev, residual norms ||A v - lambda v|| / ||v||)."""
    Al, Vl, el = A.astype(dtype), V.astype(dtype), ev.astype(dtype)
    R = Al @ Vl - Vl * el[None, :]
    vv = np.sum(Vl * Vl, axis=0)
    resid = np.sqrt(np.asarray(np.sum(R * R, axis=0) / vv, dtype=np.float64))
    m = len(ev)
    if window <= 0:
        return np.asarray(el + np.sum(Vl * R, axis=0) / vv, dtype=np.float64), resid
    bw = 2 * window
    # B[j, d + bw] = v_{j+d}^T r_j, G[j, d + bw] = v_{j+d}^T v_j
    B = np.zeros((m, 2 * bw + 1), dtype=dtype)
    G = np.zeros((m, 2 * bw + 1), dtype=dtype)
    for d in range(-bw, bw + 1):
        j = np.arange(max(0, -d), min(m, m - d))
        if len(j):
            B[j, d + bw] = np.sum(Vl[:, j + d] * R[:, j], axis=0)
            G[j, d + bw] = np.sum(Vl[:, j + d] * Vl[:, j], axis=0)
    out = np.empty(m)
    for j in range(m):
        lo, hi = max(0, j - window), min(m - 1, j + window)
        idx = np.arange(lo, hi + 1)
        kk, ll = np.meshgrid(idx, idx, indexing="ij")
        mkl = B[ll, kk - ll + bw] + el[ll] * G[ll, kk - ll + bw]
        nrm = np.sqrt(G[kk, bw] * G[ll, bw])
        M = np.asarray((0.5 * (mkl + mkl.T)) / nrm, dtype=np.float64)
        out[j] = np.sort(jacobi_eigvals(M))[j - lo]
    return out, resid


def diag_hd(hcc, scc, lch, ns, ks, itype=0, ilzero=1, ibzero=1, Edmax=0.0, Egap=0.001,
            want_vectors=False, refine=False, lowest=None, refine_dtype=np.longdouble):
    """Solve H c = E S c the way bsr_hd does for one partial wave.

    hcc, scc: (nch(nch+1)/2, ns, ns) lower-triangle channel blocks [row, col]
    as written by Record_matrix (record_matrix.f90:2).  With a block-diagonal
    S (diag_ovl /= 0) the reference solves a standard problem after the
    per-channel pre-diagonalisation (diag_hd.f90:68-71); with off-diagonal
    overlap blocks (diag_ovl = 0) it transforms them to the channel basis,
    C = I + bb_i^T S_ij bb_j (:127-186), and runs DPOTRF(C), DSYGST(1,'L') of A
    (:268-284), DSYEV, and the back-transform DTRSM('Left','L','T') (:322-334);
    so does this restatement ("generalized" in the result is True then).
    Returns dict(eval, khm, bval, ipsol, [a_vectors]).

    refine=True restates the library's refined form: the diagonal blocks of A
    are bb_i^T H_ii bb_i (diag(bval) in exact arithmetic, diag_hd.f90:188-219)
    and every eigenvalue is replaced by its windowed Rayleigh-Ritz value in refine_dtype
    (rayleigh_refine); the eigenvectors come from LAPACK DSYEV as in the
    reference (:312), or, with lowest=m, from DSYEVR for the m lowest pairs
    only (the refinement makes the result independent of the driver).  Also
    returns "a" (the symmetric A) and "resid".
    """
    from scipy.linalg import lapack

    nch = len(lch)
    blk = lambda i, j: hcc[i * (i + 1) // 2 + j]   # 0-based i >= j
    sblk = lambda i, j: scc[i * (i + 1) // 2 + j]
    gen = any(np.any(sblk(i, j) != 0) for i in range(nch) for j in range(i))
    bb = []
    bval = []
    ipsol = [0]
    for ich in range(nch):
        l = lch[ich]
        if l > ks - 2:
            l = ks - 2
        if ilzero == 0:
            l = 0
        i1 = l + 2
        i2 = ns - ibzero if itype == -1 else ns
        aa = blk(ich, ich)[i1 - 1: i2, i1 - 1: i2].copy()
        cc = sblk(ich, ich)[i1 - 1: i2, i1 - 1: i2].copy()
        w, v, info = lapack.dsygv(aa, cc, itype=1, jobz="V", uplo="U")[:3]
        if info != 0:
            raise RuntimeError("BSR_HD: channel diagonalization failed, channel %d" % (ich + 1))
        keep = np.ones(len(w), dtype=bool)
        if Edmax != 0.0:
            keep &= ~(w > Edmax)
        if Egap > 0.0:
            keep &= ~(np.abs(w) < Egap)
        vv = np.zeros((ns, int(keep.sum())))
        vv[i1 - 1: i2, :] = v[:, keep]
        bb.append(vv)
        bval.extend(w[keep].tolist())
        ipsol.append(ipsol[-1] + int(keep.sum()))
    khm = ipsol[-1]
    a = np.zeros((khm, khm), order="F")
    if not refine:
        a[np.arange(khm), np.arange(khm)] = bval
    for ic in range(nch):
        for jc in range(ic + 1 if refine else ic):
            h = blk(ic, jc)
            if not np.any(h != 0):
                continue
            w = bb[ic].T @ h          # rows: solutions of ic, cols: B-splines
            a[ipsol[ic]: ipsol[ic + 1], ipsol[jc]: ipsol[jc + 1]] = w @ bb[jc]
    out = {"khm": khm, "bval": np.array(bval), "ipsol": np.array(ipsol), "bb": bb, "generalized": gen}
    Lc = None
    if gen:
        from scipy.linalg import solve_triangular
        cmat = np.eye(khm, order="F")
        for ic in range(nch):
            for jc in range(ic):
                sij = sblk(ic, jc)
                if np.any(sij != 0):
                    cmat[ipsol[ic]: ipsol[ic + 1], ipsol[jc]: ipsol[jc + 1]] = bb[ic].T @ sij @ bb[jc]
        Lc, info = lapack.dpotrf(cmat, lower=1, clean=1)
        if info != 0:
            raise RuntimeError("BSR_HD: Cholesky factorization failed (info %d)" % info)
        a, info = lapack.dsygst(a, Lc, itype=1, lower=1)
        if info != 0:
            raise RuntimeError("DSYGST info %d" % info)
        a = np.asfortranarray(np.tril(a))
        out["c"] = np.tril(cmat) + np.tril(cmat, -1).T
        back = lambda y: solve_triangular(Lc, y, trans="T", lower=True)
    else:
        back = lambda y: y
    if refine:
        full = np.tril(a) + np.tril(a, -1).T
        if lowest is not None:
            # the Rayleigh-Ritz windows of the lowest pairs reach RR_HW pairs beyond them
            from scipy.linalg import eigh
            ev, vec = eigh(full, subset_by_index=[0, min(lowest + RR_HW, khm) - 1], driver="evr")
        else:
            ev, vec, info = lapack.dsyev(a, compute_v=1, lower=1)[:3]
            if info != 0:
                raise RuntimeError("DSYEV info %d" % info)
        ev, resid = rayleigh_refine(full, ev, vec, refine_dtype)
        if lowest is not None:
            keep = min(lowest, khm)
            ev, resid, vec = ev[:keep], resid[:keep], vec[:, :keep]
        o = np.argsort(ev, kind="stable")
        out.update({"eval": ev[o], "resid": resid[o], "vectors": back(vec[:, o]), "a": full})
        return out
    ev, vec, info = lapack.dsyev(a, compute_v=1 if want_vectors else 0, lower=1)[:3]
    if info != 0:
        raise RuntimeError("DSYEV info %d" % info)
    out["eval"] = ev
    if want_vectors:
        out["vectors"] = back(vec)
    return out


def bs_orth(basis, P, ort_lists, hcc):
    """BS_ORTH (bs_orth.f90:2-92) on host blocks hcc (nblk, ns, ns) [row, col] (the layout
    assemble returns), returned as a new array.  ort_lists: per channel, the 0-based
    orbital columns of P the channel is made orthogonal to."""
    ns, ks = basis.ns, basis.ks
    sb = np.ascontiguousarray(basis.get("sb"))          # memory = Fortran (ns, ks)
    ptr = np.zeros(len(ort_lists) + 1, dtype=np.int32)
    for i, l in enumerate(ort_lists):
        ptr[i + 1] = ptr[i] + len(l)
    idx = np.ascontiguousarray(np.concatenate([np.asarray(l, dtype=np.int32) for l in ort_lists])
                               if ptr[-1] > 0 else np.zeros(1, dtype=np.int32))
    h = np.asfortranarray(np.asarray(hcc, dtype=np.float64).transpose(1, 2, 0))   # Fortran (ns, ns, nblk)
    Pf = np.asfortranarray(P, dtype=np.float64)
    lib().orc_bs_orth(ns, ks, _p(sb), len(ort_lists), Pf.ctypes.data_as(_D), _pi(ptr), _pi(idx),
                      h.ctypes.data_as(_D))
    return h.transpose(2, 0, 1).copy()


def rsol(ns, nch, ipsol, bb, a, want_v=True):
    """rsol_out (rsol_out.f90:20-36): solutions v (nch*ns, khm) and surface amplitudes WMAT (nch, khm)."""
    ipsol = np.ascontiguousarray(ipsol, dtype=np.int32)
    khm = int(ipsol[-1])
    bbf = np.asfortranarray(bb, dtype=np.float64)
    af = np.asfortranarray(a, dtype=np.float64)
    v = np.zeros((nch * ns, khm), order="F") if want_v else None
    w = np.zeros((nch, khm), order="F")
    lib().orc_rsol(ns, nch, _pi(ipsol), bbf.ctypes.data_as(_D), khm, af.ctypes.data_as(_D),
                   v.ctypes.data_as(_D) if want_v else None, w.ctypes.data_as(_D))
    return v, w


def channel_weights(ipsol, a):
    """W_OUT (w_out.f90:58-76): wt (nch, khm), isol (khm,), iprm (nch, khm), 1-based."""
    ipsol = np.ascontiguousarray(ipsol, dtype=np.int32)
    nch, khm = len(ipsol) - 1, int(ipsol[-1])
    af = np.asfortranarray(a, dtype=np.float64)
    wt = np.zeros((nch, khm), order="F")
    isol = np.zeros(khm, dtype=np.int32)
    iprm = np.zeros((nch, khm), dtype=np.int32, order="F")
    lib().orc_channel_weights(nch, _pi(ipsol), khm, af.ctypes.data_as(_D), wt.ctypes.data_as(_D), _pi(isol),
                              _pi(iprm))
    return wt, isol, iprm


def nk(ns, ks, rkb, pi1, pj1, pi2, pj2):
    """nk.f90 (meth 'c'): N^k(i1, j1; i2, j2) from an mnk_cell table."""
    r = np.asfortranarray(rkb)
    f = [np.ascontiguousarray(x, dtype=np.float64) for x in (pi1, pj1, pi2, pj2)]
    return lib().orc_nk(ns, ks, r.ctypes.data_as(_D), r.shape[2], *[_p(x) for x in f])


def mk(ns, ks, rkb, pi1, pj1, pi2, pj2):
    """mk.f90 (meth 'c'): M^k(i1, j1; i2, j2), the rk.f90 sum over an mmk_cell table halved."""
    r = np.asfortranarray(rkb)
    f = [np.ascontiguousarray(x, dtype=np.float64) for x in (pi1, pj1, pi2, pj2)]
    return lib().orc_rk(ns, ks, r.ctypes.data_as(_D), r.shape[2], *[_p(x) for x in f]) / 2.0


def tk(ns, ks, rkb, pi1, pj1, pi2, pj2):
    """tk.f90 (meth 'c'): T^k(i1, j1; i2, j2) from an mtk_cell table."""
    r = np.asfortranarray(rkb)
    f = [np.ascontiguousarray(x, dtype=np.float64) for x in (pi1, pj1, pi2, pj2)]
    return lib().orc_tk(ns, ks, r.ctypes.data_as(_D), r.shape[2], *[_p(x) for x in f])


def vk(ns, ks, rkb, pi1, pj1, pi2, pj2):
    """vk.f90 (meth 'c'): V^k(i1, j1; i2, j2) from an mvk_cell table."""
    r = np.asfortranarray(rkb)
    f = [np.ascontiguousarray(x, dtype=np.float64) for x in (pi1, pj1, pi2, pj2)]
    return lib().orc_vk(ns, ks, r.ctypes.data_as(_D), r.shape[2], *[_p(x) for x in f])
