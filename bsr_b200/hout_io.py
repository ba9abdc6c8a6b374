"""Writers and readers of bsr_hd's output files for one partial wave.

  h.nnn     H_OUT (src/bsr/BSR_HD3/h_out.f90:2-81): the Belfast R-matrix H.DAT
            records -- target and partial-wave parameters, channel l values,
            asymptotic coefficients CF(:,:,2:lamax+1), R-matrix poles (eigenvalues)
            and surface amplitudes WMAT, poles and amplitudes in descending order
            when ihout = 0 (:71-77);
  rsol.nnn  rsol_out (src/bsr/BSR_HD3/rsol_out.f90:12-36), written for itype = 1:
            (nhm, khm, kch, kcp, ns), the eigenvalues, then one record per
            solution with its B-spline coefficients v(1:nhm).
  w.nnn     W_OUT (src/bsr/BSR_HD3/w_out.f90:54-80): (kch, kcp, khm), then per
            solution the channel weights, the dominant channel isol, the energy,
            the outer-electron n per channel, the label and the SORTA order;
  bound.nnn / ubound.nnn
            B_OUT (src/bsr/BSR_HD3/b_out.f90:2-131): the solutions below Emax
            (at most msol) with binding energy, effective n and B-spline vector,
            then all energies; formatted, unformatted or both by iub.

The labels and the outer-electron n of each channel come from the configuration
files that the angular pipeline writes; they are arguments here.

Records use gfortran's unformatted sequential layout (4-byte length markers,
default Integer 4 bytes, Real(8) 8 bytes), as in bsrmat_io.
"""
import math
import re
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


# ---------------------------------------------------------------------------
# Fortran edit descriptors used by B_OUT: Iw, Fw.d, Ew.d and Dw.d
# ---------------------------------------------------------------------------

def fmt_i(n, w):
    t = "%d" % n
    return t.rjust(w) if len(t) <= w else "*" * w


def fmt_f(x, w, d):
    t = "%.*f" % (d, x)
    if t.startswith("0.") and len(t) > w:
        t = t[1:]
    elif t.startswith("-0.") and len(t) > w:
        t = "-" + t[2:]
    return t.rjust(w) if len(t) <= w else "*" * w


def fmt_e(x, w, d, letter="E"):
    """Ew.d / Dw.d with the 0.ddd mantissa: 0.1234567890E+01; an exponent above 99
    drops the letter (+100), as the Fortran standard prescribes."""
    x = float(x)
    if x == 0.0:
        digits, e = "0" * d, 0
    else:
        mant, ex = ("%.*e" % (d - 1, abs(x))).split("e")
        digits, e = mant.replace(".", ""), int(ex) + 1
    ex = "%s%+03d" % (letter, e) if abs(e) <= 99 else "%+04d" % e
    t = ("-" if math.copysign(1.0, x) < 0 else "") + "0." + digits + ex
    return t.rjust(w) if len(t) <= w else "*" * w


def _fortran_float(tok):
    t = tok.strip().upper().replace("D", "E")
    m = re.fullmatch(r"([+-]?\d*\.\d*)([+-]\d+)", t)        # exponent without its letter
    return float(m.group(1) + "E" + m.group(2)) if m else float(t)


def conv_au(z, awt=0.0):
    """Conv_au (libs/ZCOM/conv_au.f90:2-47): a.u. -> cm^-1 and eV with the atomic
    weight awt, or the weight estimated from Z when awt = 0."""
    ratio, ry_cm, ry_ev = 5.485799110e-4, 109737.31568549, 13.6056917
    z = float(z)
    if awt != 0.0:
        a = float(awt)
    elif z == 1.0:
        a = 1.0
    elif z > 10.0:
        a = 2 * z + 1 + (z - 11) / 2
    elif int(z) % 2 == 0 or z == 7.0:
        a = 2 * z
    else:
        a = 2 * z + 1
    return 2 * ry_cm * a / (a + ratio), 2 * ry_ev * a / (a + ratio)


def bound_states(eval_, isol, iptar, etarg, nz, nelc, emax=0.0, msol=100):
    """b_out.f90:38-66: which solutions are written and their binding energies.
    isol: 1-based dominant channel per solution (channel_weights); iptar: 1-based
    target of each channel.  Returns (keep, ebind, eff_n, n_eff) over the first ms
    solutions; n_eff is -1 for a solution that is not written."""
    eval_ = np.asarray(eval_, dtype=np.float64)
    khm, kch = len(eval_), len(iptar)
    zion = float(nz - nelc)
    if zion == 0.0:
        zion = 1.0
    ms = msol if 0 < msol <= khm else khm
    ebind, eff_n = np.zeros(ms), np.zeros(ms)
    n_eff = np.full(ms, -1, dtype=np.int64)
    for i in range(ms):
        if eval_[i] > emax and emax != 0.0:
            continue
        ich = int(isol[i])
        if ich <= kch:
            it = int(iptar[ich - 1])
            ebind[i] = eval_[i] - etarg[it - 1]
            if ebind[i] > 0.0:
                n_eff[i] = ord("k") - ord("1") + 1
                eff_n[i] = math.sqrt(2 * ebind[i])
            else:
                eff_n[i] = zion / math.sqrt(abs(2 * ebind[i]))
                n_eff[i] = ord("n") - ord("1") + 1
        else:
            n_eff[i] = -2
    return n_eff != -1, ebind, eff_n, n_eff


def _label64(label):
    b = label.encode("ascii")[:64]
    return b + b" " * (64 - len(b))


def write_w(path, wt, isol, eval_, n_eff_ch, labels, iprm):
    """w.nnn as W_OUT writes it (kcp = 0): wt, iprm (kch, khm); n_eff_ch (kch, khm)
    the outer-electron n per channel; labels: the dominant channel's label per solution."""
    wt = np.asarray(wt, dtype=np.float64)
    kch, khm = wt.shape
    n_eff_ch = np.asarray(n_eff_ch, dtype=np.int32).reshape(kch, khm)
    iprm = np.asarray(iprm, dtype=np.int32).reshape(kch, khm)
    with open(path, "wb") as f:
        _rec(f, struct.pack("<3i", kch, 0, khm))
        for i in range(khm):
            _rec(f, wt[:, i].astype("<f8").tobytes() + struct.pack("<id", int(isol[i]), float(eval_[i])) +
                 n_eff_ch[:, i].astype("<i4").tobytes() + _label64(labels[i]) + iprm[:, i].astype("<i4").tobytes())


def read_w(path):
    with open(path, "rb") as f:
        kch, kcp, khm = struct.unpack("<3i", _read_rec(f))
        nw = kch + kcp
        out = {"kch": kch, "kcp": kcp, "khm": khm, "wt": np.zeros((nw, khm)), "isol": np.zeros(khm, np.int32),
               "eval": np.zeros(khm), "n_eff": np.zeros((kch, khm), np.int32), "labels": [],
               "iprm": np.zeros((nw, khm), np.int32)}
        for i in range(khm):
            r = _read_rec(f)
            o = 8 * nw
            out["wt"][:, i] = np.frombuffer(r[:o], dtype="<f8")
            out["isol"][i], out["eval"][i] = struct.unpack("<id", r[o:o + 12])
            o += 12
            out["n_eff"][:, i] = np.frombuffer(r[o:o + 4 * kch], dtype="<i4")
            o += 4 * kch
            out["labels"].append(r[o:o + 64].decode("ascii").rstrip())
            out["iprm"][:, i] = np.frombuffer(r[o + 64:o + 64 + 4 * nw], dtype="<i4")
    return out


def write_bound(path_b, path_ub, ns, eval_, v, isol, iptar, etarg, nz, nelc, lpar, ispar, ipar, labels=None,
                n_eff_ch=None, emax=0.0, msol=100, iub=-1, awt=0.0):
    """B_OUT (b_out.f90:2-131), kcp = 0.  v: solutions in the B-spline basis
    (kch*ns, khm) from rsol_out; isol from channel_weights; labels / n_eff_ch
    (kch, khm) as recorded in w.nnn (blank and 0 when absent).  iub < 0 writes
    bound.nnn only, iub > 0 ubound.nnn only, iub = 0 both (with the reference's
    record set: the vectors and energies go to ubound.nnn only when iub > 0)."""
    eval_ = np.asarray(eval_, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    nhm, khm = v.shape
    kch = len(iptar)
    if labels is None:
        labels = [""] * khm
    n_eff_ch = np.zeros((kch, khm), np.int64) if n_eff_ch is None else np.asarray(n_eff_ch).reshape(kch, khm)
    au_ev = conv_au(nz, awt)[1]
    keep, ebind, eff_n, _ = bound_states(eval_, isol, iptar, etarg, nz, nelc, emax, msol)
    nbound = int(keep.sum())
    fb = open(path_b, "w") if iub <= 0 else None
    fu = open(path_ub, "wb") if iub >= 0 else None
    try:
        if fb:
            head = "".join(fmt_i(x, 10) for x in (ns, kch, 0, nhm, nbound)) + \
                "".join(fmt_i(x, 5) for x in (lpar, ispar, ipar))
            fb.write(head.ljust(73) + "=> ns,kch,kcp,nhm,nbound,lpar,ispar,ipar\n")
        if fu:
            _rec(fu, struct.pack("<8i", ns, kch, 0, nhm, nbound, lpar, ispar, ipar))
        js = 0
        for i in range(len(keep)):
            if not keep[i]:
                continue
            js += 1
            nn = [int(x) for x in n_eff_ch[:, i]]
            if fb:
                fb.write(fmt_i(js, 5) + "  " + labels[i].rstrip() + "\n")
                fb.write(fmt_e(eval_[i], 20, 10) + fmt_f(ebind[i] * au_ev, 15, 5) + fmt_f(eff_n[i], 10, 2) +
                         "".join(fmt_i(x, 5) for x in nn) + "\n")
            if fu:
                _rec(fu, struct.pack("<i", js) + _label64(labels[i]))
                _rec(fu, struct.pack("<3d", eval_[i], ebind[i] * au_ev, eff_n[i]) + np.asarray(nn, "<i4").tobytes())
            if fb:
                col = v[:, i]
                for q in range(0, nhm, 5):
                    fb.write("".join(fmt_e(x, 15, 8, "D") for x in col[q:q + 5]) + "\n")
            if fu and iub > 0:
                _rec(fu, v[:, i].astype("<f8").tobytes())
        if fb:
            fb.write("\n" + "khm =" + fmt_i(khm, 8) + "\n\n")
            for e in eval_:
                fb.write(fmt_e(e, 16, 8, "D") + fmt_e((e - etarg[0]) * 2, 16, 8, "D") + "\n")
        if fu and iub > 0:
            for e in eval_:
                _rec(fu, struct.pack("<2d", e, (e - etarg[0]) * 2))
    finally:
        if fb:
            fb.close()
        if fu:
            fu.close()
    return nbound


def read_bound(path):
    """bound.nnn as the reference's readers take it (BSR_UTILS/bound_bsw.f90:237-263):
    list-directed header and energy lines, vectors in (5D15.8)."""
    with open(path) as f:
        lines = f.read().split("\n")
    hd = [int(x) for x in lines[0].split()[:8]]
    ns, kch, kcp, nhm, nbound, lpar, ispar, ipar = hd
    states, p = [], 1
    nrow = (nhm + 4) // 5
    for _ in range(nbound):
        js, label = int(lines[p][:5]), lines[p][7:]
        tok = lines[p + 1].split()
        e, eb, neff = (_fortran_float(x) for x in tok[:3])
        nn = [int(x) for x in tok[3:3 + kch]]
        vals = []
        for r in lines[p + 2:p + 2 + nrow]:
            vals += [_fortran_float(r[q:q + 15]) for q in range(0, len(r), 15) if r[q:q + 15].strip()]
        states.append({"js": js, "label": label, "eval": e, "ebind_ev": eb, "eff_n": neff, "n_eff": nn,
                       "v": np.array(vals)})
        p += 2 + nrow
    khm = int(lines[p + 1].split("=")[1])
    en = np.array([[_fortran_float(l[:16]), _fortran_float(l[16:32])] for l in lines[p + 3:p + 3 + khm]])
    return {"ns": ns, "kch": kch, "kcp": kcp, "nhm": nhm, "nbound": nbound, "lpar": lpar, "ispar": ispar,
            "ipar": ipar, "states": states, "khm": khm, "energies": en}

