"""The digit arithmetic of bsrg_dgemm_ozaki restated in numpy (no GPU): each row of A
and column of B scaled by a power of two below its largest magnitude, cut into S
signed 7-bit digits, the digit products of level t + u < S summed exactly in
integers and recombined in FP64 -- the scheme of tc_ozaki.cu (Ozaki, Ogita, Oishi,
Rump 2012, integer form).  Checks that every splitting step is exact, that the
digits fit int8, that the int32 accumulators cannot overflow up to k = 16384, and
the error bound the GPU tests use: 2^-(7S-6) k max|A(i,:)| max|B(:,j)|."""
import numpy as np
import pytest

KMAX = 16384            # BSRG_OZAKI_KMAX


def line_exponents(X):
    """e per row with max |x| < 2^e (frexp), 0 for an all-zero row."""
    mx = np.max(np.abs(X), axis=1)
    e = np.zeros(X.shape[0], dtype=np.int64)
    nz = mx > 0
    e[nz] = np.frexp(mx[nz])[1]
    return e


def digits(X, S):
    e = line_exponents(X)
    v = np.ldexp(X, -e[:, None])
    assert np.all(np.abs(v) < 1.0)
    planes = []
    for _ in range(S):
        y = v * 128.0
        d = np.trunc(y)
        v = y - d
        assert np.all(np.abs(d) <= 127)
        planes.append(d.astype(np.int64))
    return e, planes, v


def ozaki(A, B, S=8):
    ea, QA, _ = digits(A, S)
    eb, QB, _ = digits(B.T.copy(), S)
    acc = [np.zeros((A.shape[0], B.shape[1]), dtype=np.int64) for _ in range(S)]
    for t in range(S):
        for u in range(S - t):
            acc[t + u] += QA[t] @ QB[u].T
    for L in range(S):
        assert np.all(np.abs(acc[L]) < 2 ** 31)
    s = np.zeros(acc[0].shape)
    for L in range(S - 1, -1, -1):
        s += np.ldexp(acc[L].astype(np.float64), -7 * (L + 2))
    return np.ldexp(s, ea[:, None] + eb[None, :])


def test_splitting_is_exact():
    rng = np.random.default_rng(0)
    X = rng.standard_normal((50, 300)) * np.exp2(rng.uniform(-40, 40, (50, 1)))
    for S in (6, 7, 8):
        e, planes, r = digits(X, S)
        back = sum(np.ldexp(p.astype(np.float64), -7 * (t + 1)) for t, p in enumerate(planes))
        # x 2^-e = sum of the digits + the remainder, exactly; the remainder is below 2^-7S
        assert np.array_equal(back + np.ldexp(r, -7 * S), np.ldexp(X, -e[:, None]))
        assert np.all(np.abs(r) < 1.0)


def test_accumulators_fit_int32_at_kmax():
    # level L sums min(L+1, S) digit products of |q| <= 127 over k terms
    assert 8 * KMAX * 127 * 127 < 2 ** 31
    assert 8 * (KMAX + 2048) * 127 * 127 >= 2 ** 31 - 2 ** 27   # the limit is not far from necessary


@pytest.mark.parametrize("S", [6, 7, 8])
def test_error_bound(S):
    rng = np.random.default_rng(S)
    m, n, k = 60, 40, 900
    A = rng.standard_normal((m, k)) * np.exp2(rng.uniform(-30, 30, (m, 1)))
    B = rng.standard_normal((k, n)) * np.exp2(rng.uniform(-10, 10, (1, n)))
    C = ozaki(A, B, S)
    ref = A @ B
    bound = 2.0 ** -(7 * S - 6) * k * np.outer(np.abs(A).max(1), np.abs(B).max(0)) + 4 * 2.0 ** -52 * np.abs(ref)
    assert np.all(np.abs(C - ref) <= bound)
    if S == 8:
        assert np.max(np.abs(C - ref)) / np.max(np.abs(ref)) < 1e-14


def test_zero_lines_and_integers_exact():
    """Integer matrices with small entries are multiplied exactly, and a zero row or column
    gives exact zeros."""
    rng = np.random.default_rng(4)
    A = rng.integers(-1000, 1000, (30, 200)).astype(np.float64)
    B = rng.integers(-1000, 1000, (200, 20)).astype(np.float64)
    A[5] = 0.0
    C = ozaki(A, B, 8)
    assert np.array_equal(C, A @ B)
    assert np.all(C[5] == 0.0)
