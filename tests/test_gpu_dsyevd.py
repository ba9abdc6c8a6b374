"""bsrg_dsyevd (two-stage reduction, divide and conquer, back-transformation)
against numpy's eigh on the host: eigenvalues within 8 n eps ||A||, residual
||A Z - Z W|| and orthogonality ||Z^T Z - I|| at the same scale.  Matrices:
random symmetric (sizes across the panel width 32 and the leaf size 64),
graded (1e-3 .. 1e7 on the diagonal, like the kinetic part of H), block
diagonal (zero panels: reflectors with tau = 0), and diagonal."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
EPS = np.finfo(float).eps


def _cases():
    rng = np.random.default_rng(21)
    out = []
    for n in (1, 2, 3, 31, 33, 40, 57, 64, 97, 300, 1000, 2047):
        M = rng.standard_normal((n, n))
        out.append(("random%d" % n, (M + M.T) / 2))
    n = 800
    M = rng.standard_normal((n, n)) * 0.1
    A = (M + M.T) / 2
    A[np.arange(n), np.arange(n)] = np.logspace(-3, 7, n) * rng.choice([-1.0, 1.0], n)
    out.append(("graded", A))
    B = np.zeros((400, 400))
    for s in range(0, 400, 100):
        M = rng.standard_normal((100, 100))
        B[s:s + 100, s:s + 100] = (M + M.T) / 2
    out.append(("block-diagonal", B))
    out.append(("diagonal", np.diag(rng.standard_normal(150))))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_dsyevd(case):
    import torch
    import bsr_b200 as bsr
    from bsr_b200._lib import call
    from bsr_b200.core import _ptr
    name, A = case
    n = len(A)
    ctx = bsr.Context()
    dA = torch.from_numpy(np.tril(A).T.copy()).cuda()      # column-major, lower triangle only
    w = torch.empty(n, dtype=torch.float64, device="cuda")
    Z = torch.empty(n * n, dtype=torch.float64, device="cuda")
    call("bsrg_dsyevd", ctx.handle, n, _ptr(dA), n, _ptr(w), _ptr(Z), n)
    torch.cuda.synchronize()
    W = w.cpu().numpy()
    V = Z.cpu().numpy().reshape(n, n).T
    wr = np.linalg.eigvalsh(A)
    an = max(np.max(np.abs(wr)), 1e-300)
    tol = 8 * max(n, 16) * EPS
    assert np.all(np.diff(W) >= 0), name
    assert np.max(np.abs(W - wr)) <= tol * an, (name, np.max(np.abs(W - wr)) / an)
    R = A @ V - V * W[None, :]
    assert np.max(np.abs(R)) <= tol * an, (name, np.max(np.abs(R)) / an)
    assert np.max(np.abs(V.T @ V - np.eye(n))) <= tol, (name, np.max(np.abs(V.T @ V - np.eye(n))))
    ctx.close()


@pytest.mark.parametrize("case", [c for c in _cases() if c[0] in ("random33", "random300", "random2047", "graded",
                                                                    "block-diagonal")], ids=lambda c: c[0])
def test_dsytrd_2stage(case):
    """The reduction alone (dense -> band -> tridiagonal): T has A's eigenvalues."""
    import torch
    import bsr_b200 as bsr
    from bsr_b200._lib import call
    from bsr_b200.core import _ptr
    name, A = case
    n = len(A)
    ctx = bsr.Context()
    dA = torch.from_numpy(np.tril(A).T.copy()).cuda()
    d = torch.empty(n, dtype=torch.float64, device="cuda")
    e = torch.empty(max(n - 1, 1), dtype=torch.float64, device="cuda")
    call("bsrg_dsytrd_2stage", ctx.handle, n, _ptr(dA), n, _ptr(d), _ptr(e))
    torch.cuda.synchronize()
    dd, ee = d.cpu().numpy(), e.cpu().numpy()[: n - 1]
    T = np.diag(dd) + np.diag(ee, 1) + np.diag(ee, -1)
    wr = np.linalg.eigvalsh(A)
    an = np.max(np.abs(wr))
    assert np.max(np.abs(np.linalg.eigvalsh(T) - wr)) <= 8 * max(n, 16) * EPS * an, name
    ctx.close()


def test_dsyevd_size_sweep():
    """Every size from 1 to 300 in steps of 7, plus the panel, leaf and merged-reflector
    boundaries (32, 64, 128, 256, 257 and one more): eigenvalues, residuals and orthogonality
    at the same bar, one context reused across sizes (the workspace only grows)."""
    import torch
    import bsr_b200 as bsr
    from bsr_b200._lib import call
    from bsr_b200.core import _ptr
    rng = np.random.default_rng(5)
    ctx = bsr.Context()
    sizes = sorted(set(range(1, 301, 7)) | {32, 63, 64, 65, 128, 129, 256, 257, 258, 289})
    for n in sizes:
        M = rng.standard_normal((n, n))
        A = (M + M.T) / 2
        dA = torch.from_numpy(np.tril(A).T.copy()).cuda()
        w = torch.empty(n, dtype=torch.float64, device="cuda")
        Z = torch.empty(n * n, dtype=torch.float64, device="cuda")
        call("bsrg_dsyevd", ctx.handle, n, _ptr(dA), n, _ptr(w), _ptr(Z), n)
        torch.cuda.synchronize()
        W = w.cpu().numpy()
        V = Z.cpu().numpy().reshape(n, n).T
        wr = np.linalg.eigvalsh(A)
        an = max(np.max(np.abs(wr)), 1e-300)
        tol = 8 * max(n, 16) * EPS
        assert np.max(np.abs(W - wr)) <= tol * an, (n, np.max(np.abs(W - wr)) / an)
        assert np.max(np.abs(A @ V - V * W[None, :])) <= tol * an, n
        assert np.max(np.abs(V.T @ V - np.eye(n))) <= tol, n
    ctx.close()
