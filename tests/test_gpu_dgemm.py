"""The library's FP64 tensor-core GEMM (bsrg_dgemm, DMMA m8n8k4) against numpy
FP64 on the host: every transpose combination, ragged edges (sizes not multiples
of the 128 x 128 x 16 tile), odd leading dimensions, strided batches, beta != 0.
Tolerance: |C - C_ref| <= 8 k eps (|A||B|) elementwise (summation order differs)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
EPS = np.finfo(float).eps


def _run(ta, tb, m, n, k, batch=1, lda_pad=0, alpha=1.3, beta=0.0, seed=0):
    import torch
    from bsr_b200._lib import call
    from bsr_b200.core import _ptr, _stream
    rng = np.random.default_rng(seed)
    ar, ac = (k, m) if ta == "T" else (m, k)
    br, bc = (n, k) if tb == "T" else (k, n)
    lda, ldb, ldc = ar + lda_pad, br + lda_pad, m + lda_pad
    A = rng.standard_normal((batch, ac, lda))          # memory: batch x columns x ld (column-major per item)
    B = rng.standard_normal((batch, bc, ldb))
    C = rng.standard_normal((batch, n, ldc))
    dA, dB, dC = (torch.from_numpy(x.copy()).cuda() for x in (A, B, C))
    call("bsrg_dgemm", ta.encode(), tb.encode(), m, n, k, alpha, _ptr(dA), lda, ac * lda, _ptr(dB), ldb, bc * ldb,
         beta, _ptr(dC), ldc, n * ldc, batch, _stream())
    torch.cuda.synchronize()
    got = dC.cpu().numpy()
    for b in range(batch):
        Am = A[b, :, :ar].T           # (ar, ac) column-major view -> logical matrix
        Bm = B[b, :, :br].T
        opA = Am.T if ta == "T" else Am
        opB = Bm.T if tb == "T" else Bm
        ref = alpha * opA @ opB + beta * C[b, :, :m].T
        bound = 8 * k * EPS * (np.abs(alpha) * np.abs(opA) @ np.abs(opB) + abs(beta) * np.abs(C[b, :, :m].T)) + 1e-300
        g = got[b, :, :m].T
        assert np.all(np.abs(g - ref) <= bound), (ta, tb, m, n, k, b, np.max(np.abs(g - ref) / bound))
        # padding rows of C untouched
        if lda_pad:
            assert np.array_equal(got[b, :, m:], C[b, :, m:])


@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("tb", ["N", "T"])
def test_transposes_ragged(ta, tb):
    _run(ta, tb, 131, 77, 45)
    _run(ta, tb, 256, 128, 16)


def test_odd_leading_dims_and_beta():
    _run("N", "N", 200, 200, 200, lda_pad=3, beta=-0.7)
    _run("T", "N", 200, 200, 200, lda_pad=1, beta=1.0)


def test_strided_batch():
    _run("N", "N", 200, 200, 200, batch=5)
    _run("T", "N", 60, 50, 70, batch=3, beta=0.5)


def test_large_k_and_tiny():
    _run("N", "N", 300, 260, 2000)
    _run("N", "N", 1, 1, 1)
    _run("N", "T", 7, 3, 0, beta=0.25)        # k = 0: C = beta C


def test_rejects_bad_leading_dimension():
    import torch
    from bsr_b200._lib import BsrgError, call
    from bsr_b200.core import _ptr, _stream
    x = torch.zeros(100, dtype=torch.float64, device="cuda")
    with pytest.raises(BsrgError):
        call("bsrg_dgemm", b"N", b"N", 10, 10, 10, 1.0, _ptr(x), 5, 0, _ptr(x), 10, 0, 0.0, _ptr(x), 10, 0, 1,
             _stream())
