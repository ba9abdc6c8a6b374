"""The host-buffer entry point (bsrg_partial_wave_solve) equals the device path."""
import numpy as np
import pytest

from bsr_b200 import workload as W
from tests.gpu_helpers import to_np

pytestmark = pytest.mark.gpu


def test_partial_wave_solve_matches_device_path():
    import bsr_b200 as bsr
    pw = W.partial_wave("config1", seed=3)
    ctx = bsr.Context()
    ev_host = bsr.partial_wave_solve(ctx, pw, want_vectors=True)
    gb = bsr.define_spline(pw["t"], pw["ks"])
    H = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"])
    res = bsr.diag_hd(ctx, gb, pw["lch"], H["hcc"], want_vectors=True)
    ev_dev = to_np(res["eval"])
    assert ev_host.shape == ev_dev.shape
    assert np.max(np.abs(ev_host - ev_dev)) <= 1e-13 * np.max(np.abs(ev_dev))


def test_repeatable():
    """Same seed twice gives the same eigenvalues (determinism check)."""
    import bsr_b200 as bsr
    pw = W.partial_wave("config1", seed=4)
    ctx = bsr.Context()
    a = bsr.partial_wave_solve(ctx, pw, want_vectors=False)
    b = bsr.partial_wave_solve(ctx, pw, want_vectors=False)
    assert np.array_equal(a, b)


def test_basis_kept_only_while_the_knots_match():
    """The context keeps the last partial wave's basis; a wave on other knots (or
    another ks) gets its own, and returning to the first grid gives the first result."""
    import bsr_b200 as bsr
    pw1 = W.partial_wave("config1", seed=7)
    pw2 = dict(pw1)
    t = np.array(pw1["t"], dtype=np.float64)
    inner = slice(pw1["ks"], len(t) - pw1["ks"])
    t[inner] = t[inner] * 0.97                   # same ns and ks, different interior knots
    pw2["t"] = t
    ctx = bsr.Context()
    a = bsr.partial_wave_solve(ctx, pw1, want_vectors=False)
    b = bsr.partial_wave_solve(ctx, pw2, want_vectors=False)
    c = bsr.partial_wave_solve(ctx, pw1, want_vectors=False)
    fresh = bsr.partial_wave_solve(bsr.Context(), pw2, want_vectors=False)
    assert np.array_equal(a, c) and np.array_equal(b, fresh)
    assert not np.array_equal(a, b)
    pw3 = W.partial_wave("config4", seed=7, nch=5)    # ks 8, ns 150
    d = bsr.partial_wave_solve(ctx, pw3, want_vectors=False)
    assert np.array_equal(d, bsr.partial_wave_solve(bsr.Context(), pw3, want_vectors=False))


def test_bsr_mat_file_round_trip(tmp_path):
    """GPU assembly -> bsr_mat.nnn (the reference's file) -> GPU diag_hd gives the same spectrum
    as solving the in-memory blocks: the file carries everything bsr_hd needs."""
    import torch

    import bsr_b200 as bsr
    from bsr_b200 import bsrmat_io as io
    pw = W.partial_wave("config1", seed=9)
    ctx = bsr.Context()
    gb = bsr.define_spline(pw["t"], pw["ks"])
    H = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"], want_s=True,
                     want_acf=True)
    ev = to_np(bsr.diag_hd(ctx, gb, pw["lch"], H["hcc"], want_vectors=False)["eval"])
    hcc = to_np(H["hcc"]).transpose(2, 0, 1)
    scc = to_np(H["scc"]).transpose(2, 0, 1)
    p = tmp_path / "bsr_mat.001"
    io.write_bsr_mat(p, scc, hcc, pw["nch"], gb.ns, to_np(H["acf"]), rmax=pw["t"][-1], etarg=pw["ech"])
    r = io.read_bsr_mat(p)
    assert r["diag_ovl"] == 1
    h2 = bsr.as_fortran(np.ascontiguousarray(r["hcc"].transpose(1, 2, 0)))
    ev2 = to_np(bsr.diag_hd(ctx, gb, pw["lch"], h2, want_vectors=False)["eval"])
    assert np.array_equal(ev, ev2)
