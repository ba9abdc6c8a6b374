"""The split-precision tensor-core product (bsrg_dgemm_tf32x3: tcgen05 kind::tf32,
operands split into two TF32 parts, FP32 accumulation in tensor memory) against
numpy FP64: |C - C_ref| <= 2^-16 ((|A| |B|)_ij + |beta C|) (FP32 accumulation)
of the magnitude the product is built from (22 significant bits per operand,
FP32 accumulation over K)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k,beta", [(128, 128, 32, 0.0), (300, 200, 100, 0.5), (2000, 820, 2000, 0.0),
                                        (5, 7, 3, -1.0), (129, 130, 33, 0.0)])
def test_tf32x3_gemm(m, n, k, beta):
    import torch
    from bsr_b200._lib import call
    from bsr_b200.core import _ptr, _stream
    rng = np.random.default_rng(m + n + k)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n))
    C = rng.standard_normal((m, n))
    dA = torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).cuda()
    dB = torch.from_numpy(np.asfortranarray(B).ravel(order="F").copy()).cuda()
    dC = torch.from_numpy(np.asfortranarray(C).ravel(order="F").copy()).cuda()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    call("bsrg_dgemm_tf32x3", m, n, k, 1.5, _ptr(dA), m, _ptr(dB), k, beta, _ptr(dC), m, _ptr(err), _stream())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    got = dC.cpu().numpy().reshape(n, m).T
    ref = 1.5 * A @ B + beta * C
    # split TF32 leaves ~2^-22 per product; the FP32 accumulation in tensor memory adds ~sqrt(k) 2^-24
    # (2.8e-6 of |A||B| measured at k = 2000): bound 2^-16
    bound = 2.0 ** -16 * (1.5 * np.abs(A) @ np.abs(B) + abs(beta) * np.abs(C)) + 1e-300
    assert np.all(np.abs(got - ref) <= bound), float(np.max(np.abs(got - ref) / bound))
    # and well beyond a single TF32 product (inputs rounded to 11 bits: ~5e-4 normwise); the
    # FP32 accumulation keeps it at FP32-GEMM quality (1.5e-5 measured at k = 2000)
    rel = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert rel < 1e-4
