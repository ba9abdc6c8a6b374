"""bsr_hd's diag_hd on the GPU against the oracle's restatement (scipy LAPACK
DSYGV / DSYEV standing in for the reference's LAPACK).

Eigenvalues are compared PER EIGENVALUE: |E_gpu - E_ref| / max(|E_ref|, 1e-3)
<= 1e-11 (the floor 1e-3 is diag_hd's Egap: channel states closer to zero are
dropped by the reference).  Both sides use the refined form: A's diagonal
blocks formed as bb^T H bb and every eigenvalue replaced by its FP64 Rayleigh
quotient (long double on the oracle side at config 1).  A raw FP64 eigensolver
-- LAPACK DSYEV included -- leaves errors of ~eps ||A|| per eigenvalue, and
||A|| ~ 4e7 here (kinetic energies of the 1e-3 a.u. first knot interval), so
raw eigenvalues agree only to ~1e-7 relative at |E| ~ 0.01; the refined ones
agree to ~1e-14.  The reference's unrefined form is checked separately,
normwise."""
import numpy as np
import pytest

from bsr_b200 import workload as W
from oracle import oracle as O
from tests.gpu_helpers import to_np

pytestmark = pytest.mark.gpu
TOL_E = 1e-11          # per eigenvalue, relative (floor 1e-3)
TOL_NORMWISE = 1e-11   # unrefined reference form, relative to max |E|


def per_eig_rel(ev, er):
    return np.abs(ev - er) / np.maximum(np.abs(er), 1e-3)


def _solve(pw, want_vectors=True, refine=True):
    import bsr_b200 as bsr
    gb = bsr.define_spline(pw["t"], pw["ks"])
    ctx = bsr.Context()
    ctx.set_refine(refine)
    H = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"], want_s=True)
    res = bsr.diag_hd(ctx, gb, pw["lch"], H["hcc"], want_vectors=want_vectors, want_bb=True)
    return gb, ctx, H, res


@pytest.fixture(scope="module")
def config1():
    pw = W.partial_wave("config1")
    gb, ctx, H, res = _solve(pw)
    hcc = to_np(H["hcc"]).transpose(2, 0, 1)
    scc = to_np(H["scc"]).transpose(2, 0, 1)
    ref = O.diag_hd(hcc, scc, pw["lch"], gb.ns, gb.ks, refine=True)
    return pw, gb, ctx, H, res, ref, hcc, scc


def test_khm_and_channel_eigenvalues(config1):
    pw, gb, ctx, H, res, ref, hcc, scc = config1
    assert res["khm"] == ref["khm"]
    ev = to_np(res["eval"])
    assert ev.shape == (ref["khm"],)
    assert np.all(np.diff(ev) >= 0)


def test_eigenvalues_per_eigenvalue_config1(config1):
    pw, gb, ctx, H, res, ref, hcc, scc = config1
    ev = to_np(res["eval"])
    rel = per_eig_rel(ev, ref["eval"])
    print("config1 per-eigenvalue relative error: max %.2e p99 %.2e median %.2e" %
          (rel.max(), np.percentile(rel, 99), np.median(rel)))
    assert np.max(rel) <= TOL_E


def test_refine_stats_config1(config1):
    """The per-pair residuals the library reports are the oracle's, to rounding; the
    corrections are of the size of the raw eigensolver's error, ~eps ||A||."""
    pw, gb, ctx, H, res, ref, hcc, scc = config1
    n = res["khm"]
    corr, resid = (to_np(x) for x in ctx.refine_stats(n))
    anorm = np.max(np.abs(ref["a"]))
    assert np.all(np.isfinite(corr)) and np.all(np.isfinite(resid))
    assert np.max(resid) < 1e-13 * anorm
    assert np.max(np.abs(corr)) < 1e3 * np.finfo(float).eps * anorm


def test_reference_form_config1():
    """Refinement off: the reference's own form (diag(bval), raw DSYEV-class solve),
    normwise against the oracle's unrefined restatement."""
    pw = W.partial_wave("config1")
    gb, ctx, H, res = _solve(pw, refine=False)
    hcc = to_np(H["hcc"]).transpose(2, 0, 1)
    scc = to_np(H["scc"]).transpose(2, 0, 1)
    er = O.diag_hd(hcc, scc, pw["lch"], gb.ns, gb.ks)["eval"]
    ev = to_np(res["eval"])
    assert np.max(np.abs(ev - er)) / np.max(np.abs(er)) < TOL_NORMWISE


def test_eigenvectors_residual_config1(config1):
    """||A v - E v|| / ||A|| for the GPU eigenvectors, with A rebuilt by the oracle in
    the GPU's channel basis signs (bases agree up to the sign of each vector)."""
    pw, gb, ctx, H, res, ref, hcc, scc = config1
    V = to_np(res["vectors"])
    ev = to_np(res["eval"])
    nch, ip, ns = pw["nch"], ref["ipsol"], gb.ns
    A = ref["a"]
    bb_gpu = to_np(res["bb"])
    for ic in range(nch):
        for q in range(ip[ic + 1] - ip[ic]):
            sgn = np.sign(bb_gpu[:, ic * ns + q] @ ref["bb"][ic][:, q])
            V[ip[ic] + q, :] *= sgn
    R = A @ V - V * ev[None, :]
    assert np.max(np.abs(R)) / np.max(np.abs(A)) < 1e-12


def test_config2_lowest_1100_per_eigenvalue():
    """Full size (khm 7810): the 1100 lowest eigenvalues per eigenvalue against the oracle
    (DSYEVR for the lowest pairs of the oracle's A, FP64 windowed Rayleigh-Ritz values), and
    sum of eigenvalues = trace(A).  The 1100 reach past the clusters near E = 0 (gaps of
    1e-3), where a plain Rayleigh quotient is off by up to 2e-10."""
    pw = W.partial_wave("config2")
    gb, ctx, H, res = _solve(pw)
    ev = to_np(res["eval"])
    assert res["khm"] > 7000
    assert np.all(np.diff(ev) >= 0)
    hcc = to_np(H["hcc"]).transpose(2, 0, 1)
    scc = to_np(H["scc"]).transpose(2, 0, 1)
    del H
    ref = O.diag_hd(hcc, scc, pw["lch"], gb.ns, gb.ks, refine=True, lowest=1100, refine_dtype=np.float64)
    assert res["khm"] == ref["khm"]
    rel = per_eig_rel(ev[:1100], ref["eval"])
    print("config2 lowest 1100 per-eigenvalue relative error: max %.2e p99 %.2e" % (rel.max(), np.percentile(rel, 99)))
    assert np.max(rel) <= TOL_E
    tr = np.trace(ref["a"])
    assert abs(ev.sum() - tr) <= 1e-12 * np.abs(np.diag(ref["a"])).sum()


def test_batched_channel_solves_match_sygvd(monkeypatch):
    """The batched channel eigensolves (potrf + batched trsm + syevBatched) and the
    per-channel sygvd path give the same refined spectrum, per eigenvalue."""
    import bsr_b200 as bsr
    pw = W.partial_wave("config1", seed=8)
    gb = bsr.define_spline(pw["t"], pw["ks"])
    ctx = bsr.Context()
    H = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"])
    a = to_np(bsr.diag_hd(ctx, gb, pw["lch"], H["hcc"], want_vectors=True)["eval"])
    monkeypatch.setenv("BSRG_CHANNEL_SYGVD", "1")
    b = to_np(bsr.diag_hd(ctx, gb, pw["lch"], H["hcc"], want_vectors=True)["eval"])
    assert a.shape == b.shape
    assert np.max(per_eig_rel(a, b)) < 1e-12


@pytest.mark.parametrize("name", ["config1", "config2"])
def test_own_channel_solves_match_library(monkeypatch, name):
    """The library's own batched channel solves (banded Cholesky, Householder, bisection,
    inverse iteration, orthogonalisation) against cuSOLVER's batched path: same khm,
    refined spectra per eigenvalue, channel eigenvalues (bval) per eigenvalue, and no
    fallback taken."""
    import bsr_b200 as bsr
    pw = W.partial_wave(name)
    gb = bsr.define_spline(pw["t"], pw["ks"])
    ctx = bsr.Context()
    H = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"])
    ra = bsr.diag_hd(ctx, gb, pw["lch"], H["hcc"], want_vectors=True, want_bb=True)
    assert ctx.channel_fallbacks() == 0
    monkeypatch.setenv("BSRG_CHANNEL_LIB", "1")
    rb = bsr.diag_hd(ctx, gb, pw["lch"], H["hcc"], want_vectors=True, want_bb=True)
    assert ra["khm"] == rb["khm"]
    a, b = to_np(ra["eval"]), to_np(rb["eval"])
    rel = per_eig_rel(a, b)
    print("%s own vs library channel solves: refined eigenvalues max rel %.2e" % (name, rel.max()))
    assert np.max(rel) < 1e-12
    # channel bases (ns x nch*ns, column q of channel i at i*ns + q): equal up to the sign of each vector
    ba, bl = to_np(ra["bb"]), to_np(rb["bb"])
    assert np.all(np.isfinite(ba))
    sg = np.sign(np.sum(ba * bl, axis=0))
    sg[sg == 0] = 1.0
    dv = np.max(np.abs(ba * sg[None, :] - bl), axis=0) / np.maximum(np.max(np.abs(bl), axis=0), 1e-300)
    print("%s channel eigenvectors: max relative difference %.2e" % (name, dv.max()))
    assert np.max(dv) < 1e-4      # eigenvector error ~ eps ||C|| / gap on both sides


def test_eigensolver_choice_config1():
    """The library's two-stage eigensolver and cuSOLVER's syevd, chosen per context, give the
    same refined spectrum per eigenvalue (config 1, khm 480), and a bad choice is rejected."""
    import bsr_b200 as bsr
    pw = W.partial_wave("config1")
    gb = bsr.define_spline(pw["t"], pw["ks"])
    ctx = bsr.Context()
    H = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"])
    out = {}
    for which in ("own", "lib", "auto"):
        ctx.set_eigensolver(which)
        out[which] = to_np(bsr.diag_hd(ctx, gb, pw["lch"], H["hcc"], want_vectors=True)["eval"])
    rel = per_eig_rel(out["own"], out["lib"])
    print("config1 own vs cuSOLVER dense eigensolver, refined: max rel %.2e" % rel.max())
    assert np.max(rel) <= TOL_E
    assert np.array_equal(out["auto"], out["lib"])       # 480 rows: below the crossover
    with pytest.raises(Exception):
        bsr._lib.call("bsrg_ctx_set_eigensolver", ctx.handle, 3)

