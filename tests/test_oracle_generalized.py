"""The oracle's generalized branch of diag_hd (off-diagonal overlap blocks:
DPOTRF, DSYGST, DSYEV, DTRSM as at diag_hd.f90:268-334) against a direct
solve of the same pencil: the eigenvalues of (A, C) in the channel basis, and
the back-transformed vectors C-orthonormal.  CPU only."""
import numpy as np
import pytest
from scipy.linalg import eigh

from oracle import oracle as O


def _problem(seed=0, nch=3, ns=24, ks=5, eps=2e-3):
    rng = np.random.default_rng(seed)
    nb = nch * (nch + 1) // 2
    hcc = np.zeros((nb, ns, ns))
    scc = np.zeros((nb, ns, ns))
    band = lambda M: np.triu(np.tril(M, ks - 1), -(ks - 1))
    S0 = band(rng.uniform(0.0, 0.1, (ns, ns)))
    S0 = S0 + S0.T + np.eye(ns) * 2.0
    for i in range(nch):
        for j in range(i + 1):
            q = i * (i + 1) // 2 + j
            if i == j:
                Hd = rng.standard_normal((ns, ns))
                hcc[q] = Hd + Hd.T + np.diag(np.linspace(-3.0, 50.0, ns))
                scc[q] = S0
            else:
                hcc[q] = 0.1 * rng.standard_normal((ns, ns))
                scc[q] = eps * band(rng.standard_normal((ns, ns)))
    return hcc, scc, [0, 1, 2][:nch], ns, ks


@pytest.mark.parametrize("refine", [False, True])
def test_generalized_branch_matches_pencil(refine):
    hcc, scc, lch, ns, ks = _problem()
    out = O.diag_hd(hcc, scc, lch, ns, ks, want_vectors=True, refine=refine, refine_dtype=np.float64)
    assert out["generalized"]
    khm, ip, bb = out["khm"], out["ipsol"], out["bb"]
    # A and C in the channel basis straight from the definitions
    A = np.zeros((khm, khm))
    C = np.eye(khm)
    nch = len(lch)
    for i in range(nch):
        for j in range(i + 1):
            q = i * (i + 1) // 2 + j
            A[ip[i]:ip[i + 1], ip[j]:ip[j + 1]] = bb[i].T @ hcc[q] @ bb[j]
            if i != j:
                C[ip[i]:ip[i + 1], ip[j]:ip[j + 1]] = bb[i].T @ scc[q] @ bb[j]
    A = np.tril(A) + np.tril(A, -1).T
    C = np.tril(C) + np.tril(C, -1).T
    w = eigh(A, C, eigvals_only=True)
    assert np.max(np.abs(out["eval"] - w)) < 1e-11 * np.max(np.abs(w))
    X = out["vectors"]
    assert np.max(np.abs(X.T @ C @ X - np.eye(khm))) < 1e-10
    assert np.max(np.abs(A @ X - C @ X * out["eval"][None, :])) < 1e-9 * np.max(np.abs(A))


def test_block_diagonal_overlap_is_standard():
    hcc, scc, lch, ns, ks = _problem(eps=0.0)
    out = O.diag_hd(hcc, scc, lch, ns, ks, want_vectors=True)
    assert not out["generalized"]
