"""Writers and readers of bsr_hd's output files for one partial wave.

  h.nnn     H_OUT (src/bsr/BSR_HD3/h_out.f90:2-81): the Belfast R-matrix H.DAT
            records -- target and partial-wave parameters, channel l values,
            asymptotic coefficients CF(:,:,2:lamax+1), R-matrix poles (eigenvalues)
            and surface amplitudes WMAT, poles and amplitudes in descending order
            when ihout = 0 (:71-77);
  rsol.nnn  rsol_out (src/bsr/BSR_HD3/rsol_out.f90:12-36), written for itype = 1:
            (nhm, khm, kch, kcp, ns), the eigenvalues, then one record per
            solution with its B-spline coefficients v(1:nhm).

Records use gfortran's unformatted sequential layout (4-byte length markers,
default Integer 4 bytes, Real(8) 8 bytes), as in bsrmat_io.
"""
import struct

import numpy as np

from .bsrmat_io import _read_rec, _rec


def write_h(path, nelc, nz, lamax, ra, etarg, ltarg, istarg, iptarg, lrgl, nspn, npty, lch, iptar, cf, eval_, wmat,
            ihout=0):
    """H_OUT.  etarg/ltarg/istarg/iptarg: per target state; lch, iptar (1-based target
    of each channel): per channel; cf (nch, nch, lamax+1); eval_ (khm,); wmat (nch, khm)."""
    lch = np.asarray(lch, dtype=np.int32)
    nchan = len(lch)
    ntarg = len(etarg)
    lrang2 = int(lch.max()) + 1
    eval_ = np.asarray(eval_, dtype=np.float64)
    wmat = np.asarray(wmat, dtype=np.float64).reshape(nchan, -1)
    khm = len(eval_)
    cf = np.asarray(cf, dtype=np.float64).reshape(nchan, nchan, -1)
    nconat = np.zeros(ntarg, dtype=np.int32)
    for it in iptar:
        nconat[int(it) - 1] += 1
    with open(path, "wb") as f:
        _rec(f, struct.pack("<5i2d", nelc, nz, lrang2, lamax, ntarg, float(ra), 0.0))
        _rec(f, np.asarray(etarg, dtype="<f8").tobytes())
        _rec(f, np.asarray(ltarg, dtype="<i4").tobytes())
        _rec(f, np.asarray(istarg, dtype="<i4").tobytes() + np.asarray(iptarg, dtype="<i4").tobytes())
        _rec(f, np.zeros(3 * lrang2, dtype="<f8").tobytes())
        _rec(f, struct.pack("<6i", lrgl, nspn, npty, nchan, khm, 0))
        _rec(f, nconat.astype("<i4").tobytes())
        _rec(f, lch.astype("<i4").tobytes())
        _rec(f, np.asfortranarray(cf[:, :, 1:lamax + 1], dtype="<f8").tobytes(order="F"))
        order = slice(None, None, -1) if ihout == 0 else slice(None)
        _rec(f, eval_[order].astype("<f8").tobytes())
        _rec(f, np.asfortranarray(wmat[:, order], dtype="<f8").tobytes(order="F"))


def read_h(path):
    """Read h.nnn as H_OUT writes it (poles and amplitudes in file order)."""
    with open(path, "rb") as f:
        nelc, nz, lrang2, lamax, nast, ra, bsto = struct.unpack("<5i2d", _read_rec(f))
        etarg = np.frombuffer(_read_rec(f), dtype="<f8").copy()
        ltarg = np.frombuffer(_read_rec(f), dtype="<i4").copy()
        ip = np.frombuffer(_read_rec(f), dtype="<i4")
        istarg, iptarg = ip[:nast].copy(), ip[nast:].copy()
        buttle = np.frombuffer(_read_rec(f), dtype="<f8").copy()
        lrgl, nspn, npty, nchan, mnp2, more = struct.unpack("<6i", _read_rec(f))
        nconat = np.frombuffer(_read_rec(f), dtype="<i4").copy()
        lch = np.frombuffer(_read_rec(f), dtype="<i4").copy()
        cf = np.frombuffer(_read_rec(f), dtype="<f8").reshape((nchan, nchan, lamax), order="F").copy()
        eval_ = np.frombuffer(_read_rec(f), dtype="<f8").copy()
        wmat = np.frombuffer(_read_rec(f), dtype="<f8").reshape((nchan, mnp2), order="F").copy()
    return {"nelc": nelc, "nz": nz, "lrang2": lrang2, "lamax": lamax, "nast": nast, "ra": ra, "bsto": bsto,
            "etarg": etarg, "ltarg": ltarg, "istarg": istarg, "iptarg": iptarg, "buttle": buttle, "lrgl": lrgl,
            "nspn": nspn, "npty": npty, "nchan": nchan, "mnp2": mnp2, "more": more, "nconat": nconat, "lch": lch,
            "cf": cf, "eval": eval_, "wmat": wmat}


def write_rsol(path, ns, kch, eval_, v, kcp=0):
    """rsol.nnn: v ((kch*ns + kcp) x khm), one record per solution."""
    eval_ = np.asarray(eval_, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    nhm, khm = v.shape
    with open(path, "wb") as f:
        _rec(f, struct.pack("<5i", nhm, khm, kch, kcp, ns))
        _rec(f, eval_.astype("<f8").tobytes())
        for i in range(khm):
            _rec(f, np.ascontiguousarray(v[:, i], dtype="<f8").tobytes())


def read_rsol(path):
    with open(path, "rb") as f:
        nhm, khm, kch, kcp, ns = struct.unpack("<5i", _read_rec(f))
        eval_ = np.frombuffer(_read_rec(f), dtype="<f8").copy()
        v = np.zeros((nhm, khm), order="F")
        for i in range(khm):
            v[:, i] = np.frombuffer(_read_rec(f), dtype="<f8")
    return {"nhm": nhm, "khm": khm, "kch": kch, "kcp": kcp, "ns": ns, "eval": eval_, "v": v}
