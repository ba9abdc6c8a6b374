"""Dense symmetric eigensolver pieces on the GPU against LAPACK (scipy).

bsrg_dsytrd replaces the DSYTRD step of DSYEV (LAP_DSYEV,
src/libs/ZCOM/LAPACK_calls.f90:54-76): same reflector convention, so d, e, tau
match LAPACK's to rounding and T has the eigenvalues of A."""
import numpy as np
import pytest
import scipy.linalg as sl
from scipy.linalg import lapack

pytestmark = pytest.mark.gpu


def _sym(n, seed, spread=10.0):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    a = (a + a.T) / 2
    a += np.diag(np.linspace(0.0, spread, n))
    return a


def _q_from_reflectors(Ar, tau):
    """Q = H(0) H(1) ... H(n-2), H(i) = I - tau_i v v^T, v(i+1) = 1, v(i+2:) = A(i+2:, i)."""
    n = Ar.shape[0]
    q = np.eye(n)
    for i in range(n - 2, -1, -1):
        v = np.zeros(n)
        v[i + 1] = 1.0
        v[i + 2:] = Ar[i + 2:, i]
        q -= tau[i] * np.outer(v, v @ q)
    return q


def _run(a):
    import torch
    from bsr_b200 import core
    ctx = core.Context()
    A = core.as_fortran(a)
    d, e, tau = core.dsytrd(ctx, A)
    torch.cuda.synchronize()
    return (d.cpu().numpy(), e.cpu().numpy(), tau.cpu().numpy(), np.asfortranarray(A.cpu().numpy()))


@pytest.mark.parametrize("n", [1, 2, 3, 5, 31, 33, 63, 64, 65, 100, 129, 300, 1000, 2100])
def test_dsytrd_matches_lapack(n):
    a = _sym(n, n)
    d, e, tau, Ar = _run(a)
    ev = np.linalg.eigvalsh(a)
    if n > 1:
        et = sl.eigh_tridiagonal(d, e, eigvals_only=True)
    else:
        et = d.copy()
    scale = np.max(np.abs(ev))
    assert np.max(np.abs(et - ev)) / scale < 1e-13
    if n > 1:
        # d, e, tau follow LAPACK's to rounding; later columns drift with the
        # summation order (the reduction is backward stable, not forward exact)
        c, dl, el, taul, info = lapack.dsytrd(np.asfortranarray(a), lower=1)
        assert info == 0
        tol = 1e-12 if n <= 65 else 1e-9
        assert np.max(np.abs(d - dl)) / scale < tol
        assert np.max(np.abs(e - el)) / scale < tol
        assert np.max(np.abs(tau - taul)) < 1e3 * tol
    if 1 < n <= 300:
        # Q from the reflectors left in A: Q T Q^T = A
        q = _q_from_reflectors(Ar, tau)
        T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
        assert np.max(np.abs(q @ T @ q.T - a)) / scale < 1e-12
        assert np.max(np.abs(q.T @ q - np.eye(n))) < 1e-12


def test_dsytrd_decoupled_columns():
    """Zero columns below the diagonal (tau = 0 reflectors) and a decoupled block."""
    n = 200
    a = _sym(n, 7)
    a[:, 50:90] = 0.0
    a[50:90, :] = 0.0
    a[np.arange(50, 90), np.arange(50, 90)] = np.arange(40) * 0.5
    d, e, tau, Ar = _run(a)
    ev = np.linalg.eigvalsh(a)
    et = sl.eigh_tridiagonal(d, e, eigvals_only=True)
    assert np.max(np.abs(et - ev)) / np.max(np.abs(ev)) < 1e-13


def test_dsytrd_repeatable():
    a = _sym(777, 3)
    r1 = _run(a)
    r2 = _run(a)
    for x, y in zip(r1, r2):
        assert np.array_equal(x, y)
