"""bsr_mat.nnn interop (record_matrix.f90:2-59, sub1.f90:110-272, read by diag_hd.f90:36-64)."""
import struct

import numpy as np
import pytest

from bsr_b200 import bsrmat_io as io


def _blocks(nch, ns, rng, zero_pair=None):
    nblk = nch * (nch + 1) // 2
    h = rng.standard_normal((nblk, ns, ns))
    if zero_pair is not None:
        i, j = zero_pair
        h[(i - 1) * i // 2 + j - 1] = 0.0
    return h


def test_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    nch, ns = 4, 7
    s = np.zeros((10, ns, ns))
    for i in range(nch):
        s[i * (i + 1) // 2 + i] = np.eye(ns)
    h = _blocks(nch, ns, rng, zero_pair=(3, 1))
    acf = rng.standard_normal((nch, nch, 3))
    p = tmp_path / "bsr_mat.001"
    io.write_bsr_mat(p, s, h, nch, ns, acf, rmax=40.0, etarg=[-1.5, -0.2], ec=-3.0)
    r = io.read_bsr_mat(p)
    assert (r["ns"], r["nch"], r["kcp"], r["mk"]) == (ns, nch, 0, 2)
    assert r["diag_ovl"] == 1 and r["diag_hm"] == 0       # S block-diagonal, H not
    assert np.array_equal(r["scc"], s)
    assert np.array_equal(r["hcc"], h)
    assert np.array_equal(r["acf"], acf)
    assert r["rmax"] == 40.0 and r["ec"] == -3.0 and list(r["etarg"]) == [-1.5, -0.2]


def test_record_layout_is_gfortran_sequential(tmp_path):
    """First records byte for byte: (ns,nch,kcp), the first diagonal block, ... and the (0,idiag) end mark."""
    nch, ns = 1, 2
    s = np.array([[[1.0, 2.0], [3.0, 4.0]]])
    h = 2 * s
    p = tmp_path / "m"
    io.write_bsr_mat(p, s, h, nch, ns, np.zeros((1, 1, 1)), rmax=1.0)
    b = p.read_bytes()
    assert b[:20] == struct.pack("<i3ii", 12, ns, nch, 0, 12)
    blk = struct.pack("<i", 32) + np.array([1.0, 3.0, 2.0, 4.0]).tobytes() + struct.pack("<i", 32)
    assert b[20:20 + 40] == blk                          # column-major (Fortran) block
    assert b[60:60 + 16] == struct.pack("<i2ii", 8, 0, 1, 8)


def test_corrupt_file_is_rejected(tmp_path):
    p = tmp_path / "bad"
    p.write_bytes(struct.pack("<i3ii", 12, 2, 1, 0, 99))
    with pytest.raises(ValueError, match="markers"):
        io.read_bsr_mat(p)
