"""The product from 8-bit digits on the tensor cores (bsrg_dgemm_ozaki: tcgen05
kind::i8, exact int32 accumulation) against numpy FP64.  With 8 digits every
element is within 2^-50 k max|A(i,:)| max|B(:,j)| + 4 eps |C| of the FP64
product (the digits dropped are of order 2^-56 of the row and column maxima per
term); 6 and 7 digits within 2^-(7S-8) k max|A(i,:)| max|B(:,j)|."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(A, B, C, alpha, beta, slices=8):
    import torch
    from bsr_b200._lib import call, lib
    from bsr_b200.core import _ptr, _stream
    m, k = A.shape
    n = B.shape[1]
    dev = lambda X: torch.from_numpy(np.asfortranarray(X).ravel(order="F").copy()).cuda()
    dA, dB, dC = dev(A), dev(B), dev(C)
    nbytes = lib().bsrg_dgemm_ozaki_work_bytes(m, n, k, slices)
    ws = torch.empty(nbytes + 256, dtype=torch.uint8, device="cuda")
    wp = (ws.data_ptr() + 255) // 256 * 256
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    call("bsrg_dgemm_ozaki", m, n, k, alpha, _ptr(dA), m, _ptr(dB), k, beta, _ptr(dC), m, slices, wp, nbytes,
         _ptr(err), _stream())
    torch.cuda.synchronize()
    return dC.cpu().numpy().reshape(n, m).T, int(err.item())


def _bound(A, B, C, alpha, beta, slices):
    k = A.shape[1]
    rowmax = np.abs(A).max(axis=1) if k else np.zeros(A.shape[0])
    colmax = np.abs(B).max(axis=0) if k else np.zeros(B.shape[1])
    ref = alpha * A @ B + beta * C
    ulp = 2.0 ** -(7 * slices - 6)
    return ref, abs(alpha) * ulp * max(k, 1) * np.outer(rowmax, colmax) + 4 * 2.0 ** -52 * (
        np.abs(ref) + abs(beta) * np.abs(C)) + 1e-300


@pytest.mark.parametrize("m,n,k,beta", [(128, 64, 32, 0.0), (300, 200, 100, 0.5), (2000, 820, 2000, 0.0),
                                        (5, 7, 3, -1.0), (129, 130, 33, 0.0), (64, 1, 4097, 1.0)])
def test_ozaki_gemm(m, n, k, beta):
    rng = np.random.default_rng(m + n + k)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n))
    C = rng.standard_normal((m, n))
    got, err = _run(A, B, C, 1.5, beta)
    assert err == 0
    ref, bound = _bound(A, B, C, 1.5, beta, 8)
    assert np.all(np.abs(got - ref) <= bound), float(np.max(np.abs(got - ref) / bound))
    # FP64 quality normwise, far beyond the split-TF32 product's ~1e-5
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-13


def test_ozaki_dynamic_range_and_zero_lines():
    """Rows of A spread over 2^-60 .. 2^60, columns of B over 2^-20 .. 2^20, one zero row
    and one zero column: the per-line power-of-two scaling keeps every element's error
    relative to its own line maxima."""
    rng = np.random.default_rng(7)
    m, n, k = 200, 150, 700
    A = rng.standard_normal((m, k)) * np.exp2(rng.uniform(-60, 60, (m, 1)))
    B = rng.standard_normal((k, n)) * np.exp2(rng.uniform(-20, 20, (1, n)))
    A[17] = 0.0
    B[:, 33] = 0.0
    C = np.zeros((m, n))
    got, err = _run(A, B, C, 1.0, 0.0)
    assert err == 0
    ref, bound = _bound(A, B, C, 1.0, 0.0, 8)
    assert np.all(np.abs(got - ref) <= bound)
    assert np.all(got[17] == 0.0) and np.all(got[:, 33] == 0.0)


@pytest.mark.parametrize("slices", [6, 7])
def test_ozaki_fewer_digits(slices):
    rng = np.random.default_rng(slices)
    A = rng.standard_normal((256, 300))
    B = rng.standard_normal((300, 128))
    C = np.zeros((256, 128))
    got, err = _run(A, B, C, 1.0, 0.0, slices)
    assert err == 0
    ref, bound = _bound(A, B, C, 1.0, 0.0, slices)
    assert np.all(np.abs(got - ref) <= bound)


def test_ozaki_repeatable():
    """Integer accumulation: the result does not depend on the order of the MMAs, so two
    calls agree bit for bit."""
    rng = np.random.default_rng(3)
    A = rng.standard_normal((300, 500))
    B = rng.standard_normal((500, 170))
    C = np.zeros((300, 170))
    g1, e1 = _run(A, B, C, 1.0, 0.0)
    g2, e2 = _run(A, B, C, 1.0, 0.0)
    assert e1 == 0 and e2 == 0 and np.array_equal(g1, g2)


def test_ozaki_non_finite_flagged_and_limits():
    from bsr_b200._lib import BsrgError, call, lib
    A = np.ones((8, 8))
    A[3, 4] = np.nan
    _, err = _run(A, np.ones((8, 8)), np.zeros((8, 8)), 1.0, 0.0)
    assert err == 2
    with pytest.raises(BsrgError, match="above"):
        call("bsrg_dgemm_ozaki", 8, 8, 20000, 1.0, 1, 8, 1, 20000, 0.0, 1, 8, 8, 1, 1 << 30, 1, None)
    with pytest.raises(BsrgError, match="workspace"):
        call("bsrg_dgemm_ozaki", 8, 8, 8, 1.0, 1, 8, 1, 8, 0.0, 1, 8, 8, 256, 16, 1, None)
    assert lib().bsrg_dgemm_ozaki_work_bytes(2000, 820, 2000, 8) > 8 * 2000 * 2000
