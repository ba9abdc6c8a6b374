"""The oracle's refined diag_hd form (CPU only).

The reference's DSYEV leaves every eigenvalue of the khm x khm matrix with an
error of order eps ||A||, and the per-channel DSYGV leaves the same in bval on
A's diagonal; at config 1 ||A|| ~ 4e7, so the raw eigenvalues are good to only
~1e-7 relative at |E| ~ 0.01.  The refined form (diagonal blocks bb^T H bb,
Rayleigh quotients in long double) removes both: the refined spectrum no longer
depends on which LAPACK driver solved the channel problems or the dense one.
That is what makes a per-eigenvalue comparison of two implementations meaningful."""
import numpy as np
import pytest
from scipy.linalg import eigh

from bsr_b200 import workload as W
from oracle import oracle as O


@pytest.fixture(scope="module")
def cfg1():
    pw = W.partial_wave("config1")
    ob = O.Basis(pw["ks"], pw["t"])
    rkb_all = np.stack([ob.mrk_cell(k) for k in range(pw["kmax"] + 1)], axis=-1)
    H = O.assemble(ob, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], np.asfortranarray(rkb_all),
                   pw["coefs"], want_s=True, want_acf=False)
    return pw, ob, H


def _rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-3)


def test_refined_form_is_driver_independent(cfg1):
    pw, ob, H = cfg1
    ref = O.diag_hd(H["hcc"], H["scc"], pw["lch"], ob.ns, ob.ks, refine=True)
    # the same partial wave with the channel problems solved by another driver (DSYGVD) and
    # the dense problem by DSYEVD, then the same refinement in FP64
    nch, ns, ks = pw["nch"], ob.ns, ob.ks
    ip, khm = ref["ipsol"], ref["khm"]
    bb = []
    for ich in range(nch):
        l = min(pw["lch"][ich], ks - 2)
        i1 = l + 2
        d = ich * (ich + 1) // 2 + ich
        w, v = eigh(H["hcc"][d][i1 - 1:, i1 - 1:], H["scc"][d][i1 - 1:, i1 - 1:], driver="gvd")
        keep = np.abs(w) >= 1e-3
        b = np.zeros((ns, int(keep.sum())))
        b[i1 - 1:, :] = v[:, keep]
        bb.append(b)
        assert b.shape[1] == ip[ich + 1] - ip[ich]
    A = np.zeros((khm, khm))
    for ic in range(nch):
        for jc in range(ic + 1):
            A[ip[ic]:ip[ic + 1], ip[jc]:ip[jc + 1]] = bb[ic].T @ H["hcc"][ic * (ic + 1) // 2 + jc] @ bb[jc]
    A = np.tril(A) + np.tril(A, -1).T
    ev, V = eigh(A, driver="evd")
    e2, _ = O.rayleigh_refine(A, ev, V, np.float64)
    assert np.max(_rel(e2, ref["eval"])) < 1e-13
    # the raw reference form is far from that
    raw = O.diag_hd(H["hcc"], H["scc"], pw["lch"], ns, ks)["eval"]
    assert np.max(_rel(raw, ref["eval"])) > 1e-10


def test_refined_residuals_small(cfg1):
    pw, ob, H = cfg1
    ref = O.diag_hd(H["hcc"], H["scc"], pw["lch"], ob.ns, ob.ks, refine=True)
    anorm = np.max(np.abs(ref["a"]))
    assert np.max(ref["resid"]) < 1e-13 * anorm
    assert np.all(np.diff(ref["eval"]) >= 0)


def test_lowest_subset_matches_full(cfg1):
    pw, ob, H = cfg1
    full = O.diag_hd(H["hcc"], H["scc"], pw["lch"], ob.ns, ob.ks, refine=True)
    low = O.diag_hd(H["hcc"], H["scc"], pw["lch"], ob.ns, ob.ks, refine=True, lowest=50,
                    refine_dtype=np.float64)
    assert np.max(_rel(low["eval"], full["eval"][:50])) < 1e-13


def test_window_removes_pair_mixing():
    """A close pair whose two vectors are rotated into each other by an angle phi: the
    plain quotients are off by gap sin^2(phi) each, the windowed Rayleigh-Ritz values
    recover the pair to rounding.  Eigenvalues of a diagonal A are known exactly; the
    window also holds eigenvalues 1e8 times larger (the graded case)."""
    lam = np.concatenate([[-0.5, 0.0900, 0.0910, 0.3], np.geomspace(1e3, 1e8, 28)])
    A = np.diag(lam)
    V = np.eye(len(lam))
    phi = 3e-4
    c, s = np.cos(phi), np.sin(phi)
    V[:, [1, 2]] = V[:, [1, 2]] @ np.array([[c, -s], [s, c]])
    ev = np.einsum("ij,ij->j", V, A @ V)          # the perturbed pairs' own quotients
    plain, _ = O.rayleigh_refine(A, ev, V, np.float64, window=0)
    win, _ = O.rayleigh_refine(A, ev, V, np.float64)
    assert np.max(np.abs(plain[1:3] - lam[1:3])) > 0.5 * 1e-3 * s * s
    assert np.max(np.abs(win - lam) / np.maximum(np.abs(lam), 1e-3)) < 1e-15


def test_jacobi_matches_lapack_on_well_scaled():
    rng = np.random.default_rng(3)
    for w in (1, 2, 9, 17):
        M = rng.normal(size=(w, w))
        M = (M + M.T) / 2
        assert np.max(np.abs(np.sort(O.jacobi_eigvals(M)) - np.linalg.eigvalsh(M))) < 1e-13
