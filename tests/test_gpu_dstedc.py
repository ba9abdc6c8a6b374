"""bsrg_dstedc (tridiagonal divide and conquer) against numpy's eigvalsh/eigh on the
host: eigenvalues within 8 n eps ||T|| (any two backward-stable solvers differ by
that much), residual ||T V - V W|| and orthogonality ||V^T V - I|| at the same scale.
Matrices: random, Wilkinson W21+ style, glued Wilkinson (tiny couplings between
copies: heavy deflation by rotation), graded 1e-3..1e7, zero couplings, a tight
cluster, sizes from 1 to 7810 (the config-2 eigenproblem's order)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
EPS = np.finfo(float).eps


def _cases():
    rng = np.random.default_rng(11)
    out = []
    for n in (1, 2, 5, 64, 65, 129, 500, 2047):
        out.append(("random%d" % n, rng.standard_normal(n), rng.standard_normal(max(n - 1, 0))))
    m = 50
    wk = np.abs(np.arange(-m, m + 1)).astype(float)
    out.append(("wilkinson", wk, np.ones(2 * m)))
    out.append(("glued", np.tile(wk, 5), np.concatenate(
        [np.concatenate([np.ones(2 * m), [1e-10]]) for _ in range(4)] + [np.ones(2 * m)])))
    n = 1000
    out.append(("graded", np.logspace(-3, 7, n) * rng.choice([-1.0, 1.0], n), 10 * rng.standard_normal(n - 1)))
    out.append(("zero-couplings", rng.standard_normal(700), np.where(rng.random(699) < 0.3, 0.0,
                                                                      rng.standard_normal(699))))
    out.append(("cluster", 1.0 + 1e-12 * rng.standard_normal(300), 1e-10 * rng.standard_normal(299)))
    out.append(("config2-size", rng.standard_normal(7810) * 100, rng.standard_normal(7809)))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_dstedc(case):
    import torch
    import bsr_b200 as bsr
    from bsr_b200._lib import call
    from bsr_b200.core import _ptr
    name, d, e = case
    n = len(d)
    ctx = bsr.Context()
    dd = torch.from_numpy(d.copy()).cuda()
    ee = torch.from_numpy(np.concatenate([e, [0.0]])).cuda()
    w = torch.empty(n, dtype=torch.float64, device="cuda")
    Z = torch.empty(n * n, dtype=torch.float64, device="cuda")
    call("bsrg_dstedc", ctx.handle, n, _ptr(dd), _ptr(ee), _ptr(w), _ptr(Z), n)
    torch.cuda.synchronize()
    W = w.cpu().numpy()
    V = Z.cpu().numpy().reshape(n, n).T          # column-major
    assert np.array_equal(dd.cpu().numpy(), d), "d must not change"
    T = np.diag(d) + np.diag(e, -1) + np.diag(e, 1)
    wr = np.linalg.eigvalsh(T)
    tn = max(np.max(np.abs(wr)), 1e-300)
    tol = 8 * max(n, 8) * EPS
    assert np.all(np.diff(W) >= 0), name
    assert np.max(np.abs(W - wr)) <= tol * tn, (name, np.max(np.abs(W - wr)) / tn)
    R = T @ V - V * W[None, :]
    assert np.max(np.abs(R)) <= tol * tn, (name, np.max(np.abs(R)) / tn)
    assert np.max(np.abs(V.T @ V - np.eye(n))) <= tol, (name, np.max(np.abs(V.T @ V - np.eye(n))))
    ctx.close()
