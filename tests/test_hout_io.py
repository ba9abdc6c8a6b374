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
