"""Host-side mirror of the reference's routines on the hot path, backed by libbsrgpu.

Names, argument meaning and error behaviour follow the Fortran routines of
jagot/bsr (src/libs/BS and src/bsr/BSR_MAT3, BSR_HD3); arrays are torch CUDA
tensors whose memory is the Fortran column-major layout of the reference's
arrays (a tensor of shape (ns, ks) here has strides (1, ns)).  A reference
'Stop' becomes a BsrgError exception.
"""
import ctypes

import numpy as np
import torch

from ._lib import BsrgError, call, lib

__all__ = ["BsrgError", "define_grid", "define_spline", "Basis", "rk_moments", "mrk_cell", "density", "convol",
           "sum_amb", "Context", "Tables", "assemble", "add_two_electron", "diag_hd", "partial_wave_solve", "fortran_empty", "as_fortran"]


# ---------------------------------------------------------------------------
# layout helpers
# ---------------------------------------------------------------------------
def fortran_empty(shape, device="cuda", dtype=torch.float64):
    """Uninitialised tensor of `shape` with column-major (Fortran) memory."""
    t = torch.empty(tuple(reversed(shape)), device=device, dtype=dtype)
    return t.permute(*reversed(range(len(shape))))


def fortran_zeros(shape, device="cuda", dtype=torch.float64):
    t = torch.zeros(tuple(reversed(shape)), device=device, dtype=dtype)
    return t.permute(*reversed(range(len(shape))))


def _is_fortran(x):
    st, sz = x.stride(), x.shape
    exp = 1
    for d in range(x.dim()):
        if sz[d] != 1 and st[d] != exp:
            return False
        exp *= sz[d]
    return True


def as_fortran(x, device="cuda"):
    """Column-major float64 CUDA tensor with the values of x (numpy or torch)."""
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(np.ascontiguousarray(x.T)).permute(*reversed(range(x.ndim)))
    x = x.to(device=device, dtype=torch.float64)
    if not _is_fortran(x):
        rev = tuple(reversed(range(x.dim())))
        x = x.permute(*rev).contiguous().permute(*rev)
    return x


def _ptr(x):
    return ctypes.c_void_p(x.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


# ---------------------------------------------------------------------------
# grid and basis: define_grid.f90, define_spline.f90
# ---------------------------------------------------------------------------
def define_grid(grid_type, ks, z, h, hmax, rmax):
    """Knot sequence of define_grid (grid_type 0: mkgrid, 1: mkgrid1).

    Returns dict(t, ns, ml, me, h) with the spline_param values the reference
    leaves in its module."""
    cap = int((rmax * z / h + 1 + ks) * 2) + 4 * ks + 64
    t = np.zeros(cap)
    ns, ml, me = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    hh = ctypes.c_double()
    call("bsrg_mkgrid", grid_type, ks, z, h, hmax, rmax, _dptr(t), cap, ctypes.byref(ns), ctypes.byref(ml),
         ctypes.byref(me), ctypes.byref(hh))
    n = ns.value
    return {"t": t[: n + ks].copy(), "ns": n, "ml": ml.value, "me": me.value, "h": hh.value, "ks": ks}


class Basis:
    """define_spline's module state, resident on the GPU (spline_grid + spline_galerkin)."""

    _WHICH = {"gr": 0, "grm": 1, "grw": 2, "bsp": 3, "bsq": 4, "bspd": 5, "sb": 6, "r1": 7, "rm1": 8, "rm2": 9,
              "rm3": 10, "db1": 11, "db2": 12, "t": 13, "bb": 14, "bs": 15}

    def __init__(self, t, ks, ml=0, me=0, h=0.0):
        t = np.ascontiguousarray(t, dtype=np.float64)
        self.ks = int(ks)
        self.ns = len(t) - self.ks
        self.nv = self.ns - self.ks + 1
        self.ml, self.me, self.h = int(ml), int(me), float(h)
        self.t = t
        handle = ctypes.c_void_p()
        call("bsrg_define_spline", self.ks, self.ns, _dptr(t), self.ml, self.me, self.h, _stream(),
             ctypes.byref(handle))
        self.handle = handle

    def free(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            torch.cuda.current_stream().synchronize()
            lib().bsrg_basis_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def get(self, name):
        """Module array `name` as a Fortran-layout CUDA tensor (gr, bsp, sb, db2, ...)."""
        ks, ns, nv = self.ks, self.ns, self.nv
        shapes = {"gr": (nv, ks), "grm": (nv, ks), "grw": (nv, ks), "bsp": (nv + 1, ks, ks),
                  "bsq": (nv + 1, ks, ks), "bspd": (nv + 1, ks, ks, 2), "t": (ns + ks,), "bb": (ns, ns),
                  "bs": (ks, ns)}
        out = fortran_empty(shapes.get(name, (ns, ks)))
        call("bsrg_basis_get", self.handle, self._WHICH[name], _ptr(out), _stream())
        return out

    def mrm(self, mm):
        """mrm.f90: <B_i|r^mm|B_j> band (ns, ks)."""
        out = fortran_empty((self.ns, self.ks))
        call("bsrg_mrm", self.handle, mm, _ptr(out), _stream())
        return out


def define_spline(t, ks, ml=0, me=0, h=0.0):
    return Basis(t, ks, ml, me, h)


# ---------------------------------------------------------------------------
# R^k tables: rk_moments.f90, mrk_cell.f90
# ---------------------------------------------------------------------------
def rk_moments(basis, k):
    """(rkd1 (ik,nv), rkd2 (ik,nv), rkd (ik,ik,nv)) for multipole k."""
    ik = basis.ks * (basis.ks + 1) // 2
    rkd1 = fortran_empty((ik, basis.nv))
    rkd2 = fortran_empty((ik, basis.nv))
    rkd = fortran_empty((ik, ik, basis.nv))
    call("bsrg_rk_moments", basis.handle, k, _ptr(rkd1), _ptr(rkd2), _ptr(rkd), _stream())
    return rkd1, rkd2, rkd


def mrk_cell(basis, k, ldp=None, out=None):
    """rkb(ns,ns,ldp,ldp) = R^k(B_i B_j; B_{i+ip-1} B_{j+jp-1}) (ldp defaults to ks)."""
    ldp = basis.ks if ldp is None else ldp
    if out is None:
        out = fortran_empty((basis.ns, basis.ns, ldp, ldp))
    call("bsrg_mrk_cell", basis.handle, k, _ptr(out), ldp, _stream())
    return out


def nk_moments(basis, k):
    """Breit-Pauli N^k cell moments (rkd1 (ik,nv), rkd2 (ik,nv), rkd (ik,ik,nv)), k >= -1."""
    ik = basis.ks * (basis.ks + 1) // 2
    rkd1 = fortran_empty((ik, basis.nv))
    rkd2 = fortran_empty((ik, basis.nv))
    rkd = fortran_empty((ik, ik, basis.nv))
    call("bsrg_nk_moments", basis.handle, k, _ptr(rkd1), _ptr(rkd2), _ptr(rkd), _stream())
    return rkd1, rkd2, rkd


def mk_moments(basis, k):
    """Breit-Pauli M^k cell moments (the N^k ones with symmetrised diagonal cells), k >= -1."""
    ik = basis.ks * (basis.ks + 1) // 2
    rkd1 = fortran_empty((ik, basis.nv))
    rkd2 = fortran_empty((ik, basis.nv))
    rkd = fortran_empty((ik, ik, basis.nv))
    call("bsrg_mk_moments", basis.handle, k, _ptr(rkd1), _ptr(rkd2), _ptr(rkd), _stream())
    return rkd1, rkd2, rkd


def mmk_cell(basis, k, fine=0.25 / 137.036 ** 2, ldp=None, out=None):
    """M^k table rkb(ns,ns,ldp,ldp) times fine (mmk_cell.f90)."""
    ldp = basis.ks if ldp is None else ldp
    if out is None:
        out = fortran_empty((basis.ns, basis.ns, ldp, ldp))
    call("bsrg_mmk_cell", basis.handle, k, float(fine), _ptr(out), ldp, _stream())
    return out


def tk_moments(basis, k):
    """Breit-Pauli T^k cell moments: rkd1, rkd2 (ks*ks, nv) and rkd (ks*ks, ks*ks, nv)."""
    jk = basis.ks * basis.ks
    rkd1 = fortran_empty((jk, basis.nv))
    rkd2 = fortran_empty((jk, basis.nv))
    rkd = fortran_empty((jk, jk, basis.nv))
    call("bsrg_tk_moments", basis.handle, k, _ptr(rkd1), _ptr(rkd2), _ptr(rkd), _stream())
    return rkd1, rkd2, rkd


def mtk_cell(basis, k, fine=0.25 / 137.036 ** 2, ldp=None, out=None):
    """T^k table rkb(ns,ns,ldp,ldp), ldp >= 2ks-1 (default), times fine/(2k+1) (mtk_cell.f90)."""
    ldp = 2 * basis.ks - 1 if ldp is None else ldp
    if out is None:
        out = fortran_empty((basis.ns, basis.ns, ldp, ldp))
    call("bsrg_mtk_cell", basis.handle, k, float(fine), _ptr(out), ldp, _stream())
    return out


def vk_moments(basis, k):
    """Breit-Pauli V^k moments: rkd1, rkd2 (ik, nv), rkd3, rkd4 (ks*ks, nv), rkd (ks*ks, ik, nv)."""
    ik, jk, nv = basis.ks * (basis.ks + 1) // 2, basis.ks * basis.ks, basis.nv
    out = [fortran_empty((ik, nv)), fortran_empty((ik, nv)), fortran_empty((jk, nv)), fortran_empty((jk, nv)),
           fortran_empty((jk, ik, nv))]
    call("bsrg_vk_moments", basis.handle, k, *[_ptr(x) for x in out], _stream())
    return out


def mvk_cell(basis, k, fine=0.25 / 137.036 ** 2, ldp=None, out=None):
    """V^k table rkb(ns,ns,ldp,ldp), ldp >= 2ks-1 (default), times fine (mvk_cell.f90)."""
    ldp = 2 * basis.ks - 1 if ldp is None else ldp
    if out is None:
        out = fortran_empty((basis.ns, basis.ns, ldp, ldp))
    call("bsrg_mvk_cell", basis.handle, k, float(fine), _ptr(out), ldp, _stream())
    return out


def wk_moments(basis, k):
    """Breit-Pauli W^k moments, layouts as vk_moments."""
    ik, jk, nv = basis.ks * (basis.ks + 1) // 2, basis.ks * basis.ks, basis.nv
    out = [fortran_empty((ik, nv)), fortran_empty((ik, nv)), fortran_empty((jk, nv)), fortran_empty((jk, nv)),
           fortran_empty((jk, ik, nv))]
    call("bsrg_wk_moments", basis.handle, k, *[_ptr(x) for x in out], _stream())
    return out


def mwk_cell(basis, k, fine=0.25 / 137.036 ** 2, ldp=None, out=None):
    """W^k table rkb(ns,ns,ldp,ldp), ldp >= 2ks-1 (default), times fine (mwk_cell.f90)."""
    ldp = 2 * basis.ks - 1 if ldp is None else ldp
    if out is None:
        out = fortran_empty((basis.ns, basis.ns, ldp, ldp))
    call("bsrg_mwk_cell", basis.handle, k, float(fine), _ptr(out), ldp, _stream())
    return out


def qk_moments(basis, k):
    """Breit-Pauli Q^k moments: rkd1..rkd4 (ks*ks, nv), rkd (ks*ks, ks*ks, nv)."""
    jk, nv = basis.ks * basis.ks, basis.nv
    out = [fortran_empty((jk, nv)) for _ in range(4)] + [fortran_empty((jk, jk, nv))]
    call("bsrg_qk_moments", basis.handle, k, *[_ptr(x) for x in out], _stream())
    return out


def mqk_cell(basis, k, fine=0.25 / 137.036 ** 2, ldp=None, out=None):
    """Q^k table rkb(ns,ns,ldp,ldp), ldp >= 2ks-1 (default), times fine (mqk_cell.f90)."""
    ldp = 2 * basis.ks - 1 if ldp is None else ldp
    if out is None:
        out = fortran_empty((basis.ns, basis.ns, ldp, ldp))
    call("bsrg_mqk_cell", basis.handle, k, float(fine), _ptr(out), ldp, _stream())
    return out


def mnk_cell(basis, k, fine=0.25 / 137.036 ** 2, ldp=None, out=None):
    """N^k table rkb(ns,ns,ldp,ldp) times fine (mnk_cell.f90); i, ip the r1 splines, r2 < r1."""
    ldp = basis.ks if ldp is None else ldp
    if out is None:
        out = fortran_empty((basis.ns, basis.ns, ldp, ldp))
    call("bsrg_mnk_cell", basis.handle, k, float(fine), _ptr(out), ldp, _stream())
    return out


# ---------------------------------------------------------------------------
# density.f90, convol.f90, sum_amb.f90
# ---------------------------------------------------------------------------
def density(ns, ks, p1, p2, type):
    cols = {"s": ks, "n": 2 * ks - 1}.get(type, ns)
    d = fortran_empty((ns, cols))
    p1, p2 = as_fortran(p1), as_fortran(p2)
    call("bsrg_density", ns, ks, _ptr(d), _ptr(p1), _ptr(p2), type.encode(), _stream())
    return d


def convol(ns, ks, d, rkb, icase, sym_i, sym_j):
    """a(ns, *) = convol of rkb with density d (band result for icase 1,2; full for 3,4).

    Entries of a band result outside the band are left zero."""
    d = as_fortran(d)
    rkb = as_fortran(rkb)
    ldp = rkb.shape[2]
    a = fortran_zeros((ns, ns))
    call("bsrg_convol", ns, ks, _ptr(a), _ptr(d), _ptr(rkb), ldp, icase, sym_i.encode(), sym_j.encode(),
         _stream())
    if icase <= 2:
        so = sym_i if icase == 1 else sym_j
        return a[:, : (ks if so == "s" else 2 * ks - 1)]
    return a


def sum_amb(ns, ks, a, b, sym):
    a, b = as_fortran(a), as_fortran(b)
    out = torch.empty(1, device="cuda", dtype=torch.float64)
    call("bsrg_sum_amb", ns, ks, _ptr(a), _ptr(b), sym.encode(), _ptr(out), _stream())
    return out


def bav(ns, ks, b, v, type, side="r"):
    """bav.f90: y = B v ('s', or 'n' with side 'r') or v B ('n', side 'l') for a band matrix."""
    b, v = as_fortran(b), as_fortran(v)
    y = torch.empty(ns, device="cuda", dtype=torch.float64)
    call("bsrg_bav", ns, ks, _ptr(b), _ptr(v), _ptr(y), type.encode(), side.encode(), _stream())
    return y


def bvmv(n, k, ar, type, x, y):
    """bvmv.f90: <x, A y> for a band array."""
    ar, x, y = as_fortran(ar), as_fortran(x), as_fortran(y)
    out = torch.empty(1, device="cuda", dtype=torch.float64)
    call("bsrg_bvmv", n, k, _ptr(ar), type.encode(), _ptr(x), _ptr(y), _ptr(out), _stream())
    return out


def quadr(basis, p1, p2, m):
    """quadr.f90: <p1 | r^m | p2>."""
    p1, p2 = as_fortran(p1), as_fortran(p2)
    out = torch.empty(1, device="cuda", dtype=torch.float64)
    call("bsrg_quadr", basis.handle, _ptr(p1), _ptr(p2), m, _ptr(out), _stream())
    return out


# ---------------------------------------------------------------------------
# bsr_mat assembly and bsr_hd diagonalisation
# ---------------------------------------------------------------------------
class Context:
    """Stream + cuBLAS/cuSOLVER handles + device workspace (bsrg_ctx)."""

    def __init__(self, device=None, stream=None):
        device = torch.cuda.current_device() if device is None else device
        self.stream = stream if stream is not None else torch.cuda.current_stream(device)
        h = ctypes.c_void_p()
        call("bsrg_ctx_create", device, ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h))
        self.handle = h

    def workspace_bytes(self):
        return lib().bsrg_ctx_workspace_bytes(self.handle)

    def use_tables(self, tables):
        """Use resident R^k tables (Tables) in assemble for their basis; None stops."""
        call("bsrg_ctx_use_tables", self.handle, tables.handle if tables is not None else None)
        self._tables = tables

    STAGES = ("rk_moments", "direct", "exchange", "one_electron", "channel_eig", "transform", "dense_eig",
              "rk_expand", "refine", "eig_band", "eig_chase", "eig_dc", "eig_q2", "eig_q1")

    def stage_flops(self):
        """Executed floating-point operations per stage since the last read (then reset)."""
        f = np.zeros(len(self.STAGES))
        call("bsrg_ctx_stage_flops", self.handle, _dptr(f), len(self.STAGES))
        return {s: float(f[i]) for i, s in enumerate(self.STAGES)}

    def set_refine(self, on=True):
        """FP64 Rayleigh-quotient refinement of diag_hd's eigenpairs (on by default)."""
        call("bsrg_ctx_set_refine", self.handle, 1 if on else 0)

    def set_precision(self, mixed=True, form="i8"):
        """FP64 (mixed=False, the default) or the mixed-precision form: the direct contraction on
        the tensor cores from 8-bit digits with exact integer accumulation (form "i8", FP64
        accuracy) or as the split-TF32 product with FP32 accumulation (form "tf32")."""
        call("bsrg_ctx_set_precision", self.handle, {"i8": 1, "tf32": 2}[form] if mixed else 0)

    def set_eigensolver(self, which="auto"):
        """diag_hd's dense eigensolver: "auto" (the library's from 7000 rows, cuSOLVER's below),
        "own" (the library's two-stage solver) or "lib" (cuSOLVER's syevd)."""
        call("bsrg_ctx_set_eigensolver", self.handle, {"auto": 0, "own": 1, "lib": 2}[which])

    def refine_stats(self, n):
        """(correction, residual norm) per eigenpair of the last refined diag_hd, as CUDA tensors."""
        corr = torch.empty(n, device="cuda", dtype=torch.float64)
        res = torch.empty(n, device="cuda", dtype=torch.float64)
        call("bsrg_diag_hd_refine_stats", self.handle, n, _ptr(corr), _ptr(res))
        return corr, res

    def channel_fallbacks(self):
        """diag_hd calls on this context whose channel solves went to the cuSOLVER fallback."""
        n = ctypes.c_int()
        call("bsrg_ctx_channel_fallbacks", self.handle, ctypes.byref(n))
        return n.value

    def set_timing(self, on=True):
        call("bsrg_ctx_set_timing", self.handle, 1 if on else 0)

    def stage_times(self):
        """Per-stage device time (ms) and launch counts since the last read (then reset)."""
        ms = np.zeros(len(self.STAGES))
        n = np.zeros(len(self.STAGES), dtype=np.int32)
        call("bsrg_ctx_stage_times", self.handle, _dptr(ms), _iptr(n), len(self.STAGES))
        return {s: (float(ms[i]), int(n[i])) for i, s in enumerate(self.STAGES)}

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            lib().bsrg_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Tables:
    """R^k tables of k = 0..kmax for one basis, resident on the device."""

    def __init__(self, ctx, basis, kmax):
        h = ctypes.c_void_p()
        call("bsrg_tables_create", ctx.handle, basis.handle, kmax, ctypes.byref(h))
        self.handle, self.basis, self.kmax = h, basis, kmax

    def nbytes(self):
        return lib().bsrg_tables_bytes(self.handle)

    def free(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            torch.cuda.synchronize()
            lib().bsrg_tables_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _coef_arrays(coefs):
    out = {k: np.ascontiguousarray(coefs[k], dtype=np.int32) for k in ("k", "type", "ich", "jch", "a", "b")}
    out["c"] = np.ascontiguousarray(coefs["c"], dtype=np.float64)
    return out


def assemble(ctx, basis, z, lch, ech, P, kmax, coefs, want_s=False, want_acf=False):
    """bsr_mat SUB1 for one partial wave: H blocks hcc (ns, ns, nch(nch+1)/2) on the device."""
    ns = basis.ns
    lch_a = np.ascontiguousarray(lch, dtype=np.int32)
    ech_a = np.ascontiguousarray(ech, dtype=np.float64)
    nch = len(lch_a)
    nblk = nch * (nch + 1) // 2
    Pd = as_fortran(P)
    c = _coef_arrays(coefs)
    hcc = fortran_empty((ns, ns, nblk))
    scc = fortran_empty((ns, ns, nblk)) if want_s else None
    acf = fortran_empty((nch, nch, kmax + 1)) if want_acf else None
    call("bsrg_assemble", ctx.handle, basis.handle, float(z), nch, _iptr(lch_a), _dptr(ech_a), Pd.shape[1],
         _ptr(Pd), kmax, len(c["c"]), _iptr(c["k"]), _iptr(c["type"]), _iptr(c["ich"]), _iptr(c["jch"]),
         _iptr(c["a"]), _iptr(c["b"]), _dptr(c["c"]), _ptr(hcc), _ptr(scc) if want_s else None,
         _ptr(acf) if want_acf else None)
    out = {"hcc": hcc}
    if want_s:
        out["scc"] = scc
    if want_acf:
        out["acf"] = acf
    return out


def add_two_electron(ctx, basis, nch, P, kmax, coefs, hcc, acf=None):
    """I_data Case(6..9) alone: accumulate the R^k groups into existing blocks hcc (and acf)."""
    Pd = as_fortran(P)
    c = _coef_arrays(coefs)
    call("bsrg_add_two_electron", ctx.handle, basis.handle, nch, Pd.shape[1], _ptr(Pd), kmax, len(c["c"]),
         _iptr(c["k"]), _iptr(c["type"]), _iptr(c["ich"]), _iptr(c["jch"]), _iptr(c["a"]), _iptr(c["b"]),
         _dptr(c["c"]), _ptr(hcc), _ptr(acf) if acf is not None else None)
    return hcc


def diag_hd(ctx, basis, lch, hcc, itype=0, ilzero=1, ibzero=1, Edmax=0.0, Egap=0.001, want_vectors=True,
            want_bb=False, scc=None):
    """bsr_hd diag_hd: eigenvalues (khm,) [+ vectors (khm,khm), bb].  With scc (the channel
    overlap blocks in hcc's layout; its off-diagonal blocks define the generalized problem,
    the diagonal ones are the basis overlap) the generalized branch runs (DPOTRF, DSYGST,
    DTRSM of diag_hd.f90:268-334); without it S is block diagonal."""
    lch_a = np.ascontiguousarray(lch, dtype=np.int32)
    nch = len(lch_a)
    ns = basis.ns
    ev = torch.empty(nch * ns, device="cuda", dtype=torch.float64)
    vecs = torch.empty((nch * ns) ** 2, device="cuda", dtype=torch.float64) if want_vectors else None
    bb = fortran_empty((ns, nch * ns)) if want_bb else None
    khm = ctypes.c_int()
    if scc is None:
        call("bsrg_diag_hd", ctx.handle, basis.handle, nch, _iptr(lch_a), _ptr(as_fortran(hcc)), itype, ilzero,
             ibzero, float(Edmax), float(Egap), 1 if want_vectors else 0, _ptr(ev), ctypes.byref(khm),
             _ptr(vecs) if want_vectors else None, _ptr(bb) if want_bb else None)
    else:
        call("bsrg_diag_hd_gen", ctx.handle, basis.handle, nch, _iptr(lch_a), _ptr(as_fortran(hcc)),
             _ptr(as_fortran(scc)), itype, ilzero, ibzero, float(Edmax), float(Egap), 1 if want_vectors else 0,
             _ptr(ev), ctypes.byref(khm), _ptr(vecs) if want_vectors else None, _ptr(bb) if want_bb else None)
    n = khm.value
    ipsol = np.zeros(nch + 1, dtype=np.int32)
    call("bsrg_diag_hd_ipsol", ctx.handle, nch, _iptr(ipsol))
    out = {"eval": ev[:n], "khm": n, "ipsol": ipsol}
    if want_vectors:
        out["vectors"] = vecs[: n * n].view(n, n).t()      # column-major (khm, khm)
    if want_bb:
        out["bb"] = bb
    return out


def dgemm(A, B, transa="N", transb="N", alpha=1.0, beta=0.0, C=None):
    """C = alpha op(A) op(B) + beta C on the FP64 tensor pipe (column-major CUDA tensors)."""
    A, B = as_fortran(A), as_fortran(B)
    m = A.shape[1] if transa == "T" else A.shape[0]
    k = A.shape[0] if transa == "T" else A.shape[1]
    n = B.shape[0] if transb == "T" else B.shape[1]
    if C is None:
        C = fortran_zeros((m, n))
    call("bsrg_dgemm", transa.encode(), transb.encode(), m, n, k, float(alpha), _ptr(A), max(1, A.stride(1)), 0,
         _ptr(B), max(1, B.stride(1)), 0, float(beta), _ptr(C), max(1, C.stride(1)), 0, 1, _stream())
    return C


def bs_orth(ctx, basis, P, ort_lists, hcc):
    """BS_ORTH on the device blocks hcc (ns, ns, nblk) in place: channel i made
    orthogonal to the orbitals (0-based columns of P) in ort_lists[i]."""
    nch = len(ort_lists)
    ptr = np.zeros(nch + 1, dtype=np.int32)
    for i, l in enumerate(ort_lists):
        ptr[i + 1] = ptr[i] + len(l)
    idx = np.ascontiguousarray(np.concatenate([np.asarray(l, dtype=np.int32) for l in ort_lists])
                               if ptr[-1] > 0 else np.zeros(1, dtype=np.int32), dtype=np.int32)
    Pd = as_fortran(P)
    call("bsrg_bs_orth", ctx.handle, basis.handle, nch, Pd.shape[1], _ptr(Pd), _iptr(ptr), _iptr(idx), _ptr(hcc))
    return hcc


def rsol_out(ctx, ns, ipsol, bb, vectors, want_v=True):
    """rsol_out: solutions in the B-spline basis v ((nch*ns) x khm) and surface amplitudes WMAT (nch x khm)."""
    ipsol = np.ascontiguousarray(ipsol, dtype=np.int32)
    nch, khm = len(ipsol) - 1, int(ipsol[-1])
    a = as_fortran(vectors)
    v = fortran_empty((nch * ns, khm)) if want_v else None
    w = fortran_empty((nch, khm))
    call("bsrg_rsol_out", ctx.handle, ns, nch, _iptr(ipsol), _ptr(as_fortran(bb)), khm, _ptr(a),
         _ptr(v) if want_v else None, _ptr(w))
    return v, w


def channel_weights(ctx, ipsol, vectors, want_iprm=True):
    """W_OUT's weights: wt (nch x khm), isol (khm,, 1-based dominant channel) and
    iprm (nch x khm, SORTA order, 1-based) of the eigenvectors a (khm x khm)."""
    ipsol = np.ascontiguousarray(ipsol, dtype=np.int32)
    nch, khm = len(ipsol) - 1, int(ipsol[-1])
    a = as_fortran(vectors)
    wt = fortran_empty((nch, khm))
    isol = torch.empty(khm, device="cuda", dtype=torch.int32)
    iprm = fortran_empty((nch, khm), dtype=torch.int32) if want_iprm else None
    call("bsrg_channel_weights", ctx.handle, nch, _iptr(ipsol), khm, _ptr(a), _ptr(wt), _ptr(isol),
         _ptr(iprm) if want_iprm else None)
    return wt, isol, iprm


def dsytrd(ctx, A):
    """LAPACK DSYTRD (lower) on the device: returns (d, e, tau); A (n x n, Fortran
    layout, overwritten) keeps the reflectors below the subdiagonal."""
    n = A.shape[0]
    d = torch.empty(max(n, 1), device="cuda", dtype=torch.float64)
    e = torch.empty(max(n - 1, 1), device="cuda", dtype=torch.float64)
    tau = torch.empty(max(n - 1, 1), device="cuda", dtype=torch.float64)
    call("bsrg_dsytrd", ctx.handle, n, _ptr(A), n, _ptr(d), _ptr(e), _ptr(tau))
    return d[:n], e[:max(n - 1, 0)], tau[:max(n - 1, 0)]


def partial_wave_solve(ctx, pw, want_vectors=True):
    """The whole path with host buffers (e2e): knots, orbitals, coefficients in; eigenvalues out."""
    t = np.ascontiguousarray(pw["t"], dtype=np.float64)
    P = np.asfortranarray(pw["P"], dtype=np.float64)
    lch = np.ascontiguousarray(pw["lch"], dtype=np.int32)
    ech = np.ascontiguousarray(pw["ech"], dtype=np.float64)
    c = _coef_arrays(pw["coefs"])
    nch, ns, ks = len(lch), len(t) - pw["ks"], pw["ks"]
    ev = np.zeros(nch * ns)
    khm = ctypes.c_int()
    call("bsrg_partial_wave_solve", ctx.handle, ks, ns, _dptr(t), float(pw["z"]), nch, _iptr(lch), _dptr(ech),
         P.shape[1], P.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), pw["kmax"], len(c["c"]), _iptr(c["k"]),
         _iptr(c["type"]), _iptr(c["ich"]), _iptr(c["jch"]), _iptr(c["a"]), _iptr(c["b"]), _dptr(c["c"]),
         1 if want_vectors else 0, _dptr(ev), ctypes.byref(khm))
    return ev[: khm.value].copy()
