"""h.nnn and rsol.nnn writers/readers (host logic; record layout of h_out.f90:2-81
and rsol_out.f90:12-36)."""
import struct

import numpy as np

from bsr_b200 import hout_io


def test_h_round_trip_and_order(tmp_path):
    rng = np.random.default_rng(0)
    nch, khm, lamax = 3, 7, 2
    ev = np.sort(rng.standard_normal(khm))
    w = rng.standard_normal((nch, khm))
    cf = rng.standard_normal((nch, nch, lamax + 1))
    p = tmp_path / "h.001"
    hout_io.write_h(p, nelc=3, nz=4, lamax=lamax, ra=20.0, etarg=[-1.0], ltarg=[0], istarg=[2], iptarg=[1],
                    lrgl=2, nspn=2, npty=1, lch=[0, 1, 2], iptar=[1, 1, 1], cf=cf, eval_=ev, wmat=w)
    h = hout_io.read_h(p)
    assert (h["nelc"], h["nz"], h["lrang2"], h["lamax"], h["nast"]) == (3, 4, 3, lamax, 1)
    assert h["ra"] == 20.0 and h["bsto"] == 0.0 and np.all(h["buttle"] == 0.0) and len(h["buttle"]) == 9
    assert (h["lrgl"], h["nspn"], h["npty"], h["nchan"], h["mnp2"], h["more"]) == (2, 2, 1, nch, khm, 0)
    assert np.array_equal(h["eval"], ev[::-1]) and np.array_equal(h["wmat"], w[:, ::-1])
    assert np.array_equal(h["cf"], cf[:, :, 1:])
    hout_io.write_h(p, nelc=3, nz=4, lamax=lamax, ra=20.0, etarg=[-1.0], ltarg=[0], istarg=[2], iptarg=[1],
                    lrgl=2, nspn=2, npty=1, lch=[0, 1, 2], iptar=[1, 1, 1], cf=cf, eval_=ev, wmat=w, ihout=1)
    h = hout_io.read_h(p)
    assert np.array_equal(h["eval"], ev) and np.array_equal(h["wmat"], w)


def test_h_first_record_layout(tmp_path):
    p = tmp_path / "h.002"
    hout_io.write_h(p, nelc=1, nz=2, lamax=0, ra=5.0, etarg=[0.0], ltarg=[0], istarg=[1], iptarg=[1], lrgl=0,
                    nspn=1, npty=0, lch=[0], iptar=[1], cf=np.zeros((1, 1, 1)), eval_=[1.0], wmat=[[0.5]])
    raw = p.read_bytes()
    n = struct.unpack("<i", raw[:4])[0]
    assert n == 5 * 4 + 2 * 8
    assert struct.unpack("<5i2d", raw[4:4 + n]) == (1, 2, 1, 0, 1, 5.0, 0.0)


def test_rsol_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    v = rng.standard_normal((12, 5))
    ev = rng.standard_normal(5)
    p = tmp_path / "rsol.001"
    hout_io.write_rsol(p, 4, 3, ev, v)
    r = hout_io.read_rsol(p)
    assert (r["nhm"], r["khm"], r["kch"], r["kcp"], r["ns"]) == (12, 5, 3, 0, 4)
    assert np.array_equal(r["v"], v) and np.array_equal(r["eval"], ev)


def test_fortran_edit_descriptors():
    """The edit descriptors of b_out.f90's formats: Ew.d / Dw.d with the 0.ddd
    mantissa, Fw.d, Iw, asterisks on overflow."""
    assert hout_io.fmt_e(1.0, 15, 8, "D") == " 0.10000000D+01"
    assert hout_io.fmt_e(-0.5, 15, 8, "D") == "-0.50000000D+00"
    assert hout_io.fmt_e(0.0, 16, 8, "D") == "  0.00000000D+00"
    assert hout_io.fmt_e(-1.2345678901e-3, 20, 10) == "   -0.1234567890E-02"
    assert hout_io.fmt_e(9.999999999e5, 15, 8, "D") == " 0.10000000D+07"
    assert hout_io.fmt_e(2.5e-120, 15, 8, "D") == " 0.25000000-119"
    assert hout_io.fmt_f(-27.2, 15, 5) == "      -27.20000"
    assert hout_io.fmt_f(3.14159, 10, 2) == "      3.14"
    assert hout_io.fmt_i(7, 5) == "    7" and hout_io.fmt_i(123456, 5) == "*****"
    for s in (" 0.10000000D+01", "-0.50000000D+00", " 0.25000000-119"):
        assert hout_io._fortran_float(s) == float(s.replace("D", "E").replace("0-119", "0E-119"))


def test_conv_au():
    """conv_au.f90: atomic weight from Z when none is given (Z = 2 -> A = 4, Z = 18 -> 40.5)."""
    r, ry_cm, ry_ev = 5.485799110e-4, 109737.31568549, 13.6056917
    for z, a in ((1, 1.0), (2, 4.0), (7, 14.0), (9, 19.0), (18, 2 * 18 + 1 + (18 - 11) / 2)):
        cm, ev = hout_io.conv_au(z)
        assert cm == 2 * ry_cm * a / (a + r) and ev == 2 * ry_ev * a / (a + r)
    assert hout_io.conv_au(2, 3.0)[1] == 2 * ry_ev * 3.0 / (3.0 + r)


def test_bound_states_selection():
    """b_out.f90:38-66: Emax cut, msol cap, binding energy against the dominant
    channel's target, effective n for closed (zion / sqrt(2|Eb|)) and open channels."""
    ev = np.array([-2.0, -1.1, -0.3, 0.2, 0.9])
    isol = np.array([1, 2, 2, 1, 2])
    iptar = [1, 2]
    etarg = [-1.0, -0.5]
    keep, eb, effn, neff = hout_io.bound_states(ev, isol, iptar, etarg, nz=3, nelc=2, emax=0.5, msol=4)
    assert list(keep) == [True, True, True, True]
    assert np.allclose(eb, [-1.0, -0.6, 0.2, 1.2])
    assert effn[0] == 1.0 / np.sqrt(2.0) and effn[2] == np.sqrt(0.4)
    assert list(neff) == [ord("n") - ord("1") + 1] * 2 + [ord("k") - ord("1") + 1] * 2
    keep, *_ = hout_io.bound_states(ev, isol, iptar, etarg, nz=3, nelc=2, emax=-0.5, msol=0)
    assert list(keep) == [True, True, False, False, False]
    _, _, effn, _ = hout_io.bound_states(ev, isol, iptar, etarg, nz=2, nelc=2)   # neutral: zion = 1
    assert effn[0] == 1.0 / np.sqrt(2.0)


def _bound_case(seed=0):
    rng = np.random.default_rng(seed)
    ns, kch, khm = 7, 3, 12
    ev = np.sort(rng.uniform(-3.0, 1.0, khm))
    v = rng.standard_normal((kch * ns, khm)) * 10.0 ** rng.integers(-30, 3, (kch * ns, khm))
    isol = rng.integers(1, kch + 1, khm)
    labels = ["state %d" % i for i in range(khm)]
    neff = rng.integers(1, 9, (kch, khm))
    return ns, kch, khm, ev, v, isol, labels, neff


def test_bound_formatted_round_trip(tmp_path):
    ns, kch, khm, ev, v, isol, labels, neff = _bound_case()
    pb, pu = tmp_path / "bound.001", tmp_path / "ubound.001"
    nb = hout_io.write_bound(pb, pu, ns, ev, v, isol, [1, 2, 1], [-1.0, -0.5], nz=3, nelc=2, lpar=1, ispar=2,
                             ipar=-1, labels=labels, n_eff_ch=neff, emax=0.5, msol=10, iub=-1)
    assert not pu.exists()
    lines = open(pb).read().split("\n")
    assert len(lines[0]) > 73 and lines[0][73:].startswith("=> ns,kch,kcp,nhm,nbound")
    r = hout_io.read_bound(pb)
    keep, eb, effn, _ = hout_io.bound_states(ev, isol, [1, 2, 1], [-1.0, -0.5], 3, 2, 0.5, 10)
    idx = np.nonzero(keep)[0]
    assert (r["ns"], r["kch"], r["kcp"], r["nhm"], r["nbound"]) == (ns, kch, 0, kch * ns, nb) and nb == len(idx)
    assert (r["lpar"], r["ispar"], r["ipar"]) == (1, 2, -1)
    au_ev = hout_io.conv_au(3)[1]
    for js, (st, i) in enumerate(zip(r["states"], idx), 1):
        assert st["js"] == js and st["label"] == labels[i] and st["n_eff"] == list(neff[:, i])
        assert abs(st["eval"] - ev[i]) <= 5e-10 * abs(ev[i])                       # E20.10: 10 digits
        assert abs(st["ebind_ev"] - eb[i] * au_ev) <= 5e-6
        assert np.all(np.abs(st["v"] - v[:, i]) <= 5e-8 * np.abs(v[:, i]))       # D15.8: 8 digits
    assert r["khm"] == khm
    assert np.all(np.abs(r["energies"][:, 0] - ev) <= 5e-8 * np.abs(ev))
    assert np.all(np.abs(r["energies"][:, 1] - (ev + 1.0) * 2) <= 5e-8 * np.abs((ev + 1.0) * 2))


def test_ubound_unformatted_records(tmp_path):
    """iub > 0: ubound.nnn only, with the vectors and the energy records; iub = 0
    writes both files and (as b_out.f90 does) no vectors into ubound.nnn."""
    from bsr_b200.bsrmat_io import _read_rec
    ns, kch, khm, ev, v, isol, labels, neff = _bound_case(1)
    pb, pu = tmp_path / "bound.002", tmp_path / "ubound.002"
    nb = hout_io.write_bound(pb, pu, ns, ev, v, isol, [1, 1, 2], [-1.0, -0.5], 4, 2, 0, 0, 1, labels=labels,
                             n_eff_ch=neff, iub=1)
    assert not pb.exists() and nb == khm
    with open(pu, "rb") as f:
        assert struct.unpack("<8i", _read_rec(f)) == (ns, kch, 0, kch * ns, nb, 0, 0, 1)
        for i in range(nb):
            r = _read_rec(f)
            assert struct.unpack("<i", r[:4])[0] == i + 1 and r[4:].decode().rstrip() == labels[i]
            r = _read_rec(f)
            assert struct.unpack("<d", r[:8])[0] == ev[i]
            assert list(np.frombuffer(r[24:], "<i4")) == list(neff[:, i])
            assert np.array_equal(np.frombuffer(_read_rec(f), "<f8"), v[:, i])
        for i in range(khm):
            assert struct.unpack("<2d", _read_rec(f)) == (ev[i], (ev[i] + 1.0) * 2)
        assert f.read() == b""
    hout_io.write_bound(pb, pu, ns, ev, v, isol, [1, 1, 2], [-1.0, -0.5], 4, 2, 0, 0, 1, iub=0)
    assert pb.exists()
    with open(pu, "rb") as f:
        _read_rec(f)
        n = 0
        while f.read(1):
            f.seek(-1, 1)
            _read_rec(f)
            n += 1
    assert n == 2 * khm


def test_w_round_trip(tmp_path):
    from oracle import oracle as O
    rng = np.random.default_rng(3)
    ipsol = np.array([0, 4, 4, 9, 15], np.int32)
    a = rng.standard_normal((15, 15))
    wt, isol, iprm = O.channel_weights(ipsol, a)
    ev = np.sort(rng.uniform(-2, 0, 15))
    neff = rng.integers(1, 6, (4, 15))
    labels = ["2s2p(3P) ch%d" % i for i in range(15)]
    p = tmp_path / "w.001"
    hout_io.write_w(p, wt, isol, ev, neff, labels, iprm)
    r = hout_io.read_w(p)
    assert (r["kch"], r["kcp"], r["khm"]) == (4, 0, 15)
    assert np.array_equal(r["wt"], wt) and np.array_equal(r["isol"], isol) and np.array_equal(r["iprm"], iprm)
    assert np.array_equal(r["eval"], ev) and np.array_equal(r["n_eff"], neff) and r["labels"] == labels
