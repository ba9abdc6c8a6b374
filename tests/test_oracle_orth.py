"""The oracle's BS_ORTH and rsol_out restatements (CPU).

BS_ORTH (src/bsr/BSR_MAT3/bs_orth.f90:2-92) applies (1 - B zz_i) on the left of
every block of channel row i and (1 - zz_j B) on the right of channel column j,
one channel after another; by associativity the result is M_i H_ij M_j^T with
M_i = 1 - B zz_i whatever the order, and for B-orthonormal orbitals the rows of
channel i become orthogonal to them."""
import numpy as np

from bsr_b200 import workload as W
from oracle import oracle as O


def _setup(nch=5, seed=3):
    cfg = W.CONFIGS["config1"]
    t, _ = W.knot_grid(cfg["ks"], cfg["ns"], cfg["rmin"], cfg["rmax"])
    ob = O.Basis(cfg["ks"], t)
    ns = ob.ns
    rng = np.random.default_rng(seed)
    nblk = nch * (nch + 1) // 2
    h = rng.standard_normal((nblk, ns, ns))
    for i in range(nch):
        d = i * (i + 1) // 2 + i
        h[d] = (h[d] + h[d].T) / 2
    B = np.zeros((ns, ns))
    sb = ob.band("sb")
    ks = ob.ks
    for jp in range(ks):
        for i in range(ks - 1 - jp, ns):
            j = i + jp - (ks - 1)
            B[i, j] = B[j, i] = sb[i, jp]
    return ob, ns, nch, h, B, rng


def _blk(i, j):
    return i * (i + 1) // 2 + j            # 0-based, i >= j


def test_bs_orth_equals_two_sided_projection():
    ob, ns, nch, h, B, rng = _setup()
    P = rng.standard_normal((ns, 6))
    lists = [[0, 2], [], [1], [3, 4, 5], []]
    got = O.bs_orth(ob, P, lists, h)
    M = []
    for l in lists:
        zz = sum((np.outer(P[:, j], P[:, j]) for j in l), np.zeros((ns, ns)))
        M.append(np.eye(ns) - B @ zz)
    scale = np.max(np.abs(h))
    for i in range(nch):
        for j in range(i + 1):
            want = M[i] @ h[_blk(i, j)] @ M[j].T
            assert np.max(np.abs(got[_blk(i, j)] - want)) / scale < 1e-12


def test_bs_orth_projects_out_orthonormal_orbitals():
    ob, ns, nch, h, B, rng = _setup(nch=4, seed=5)
    X = rng.standard_normal((ns, 3))
    L = np.linalg.cholesky(X.T @ B @ X)
    P = X @ np.linalg.inv(L).T                # P^T B P = 1
    lists = [[0, 1], [2], [], [0]]
    got = O.bs_orth(ob, P, lists, h)
    scale = np.max(np.abs(h))
    for i, l in enumerate(lists):
        for j in range(nch):
            blk = got[_blk(i, j)] if i >= j else got[_blk(j, i)].T      # channel-i rows of H(i, j)
            for q in l:
                assert np.max(np.abs(P[:, q] @ blk)) / scale < 1e-11


def test_rsol_amplitudes():
    rng = np.random.default_rng(1)
    ns, nch = 12, 3
    nsol = [10, 12, 7]
    ipsol = np.concatenate([[0], np.cumsum(nsol)]).astype(np.int32)
    khm = int(ipsol[-1])
    bb = np.zeros((ns, nch * ns))
    for ich, m in enumerate(nsol):
        bb[:, ich * ns: ich * ns + m] = rng.standard_normal((ns, m))
    a = rng.standard_normal((khm, khm))
    v, w = O.rsol(ns, nch, ipsol, bb, a)
    for ich, m in enumerate(nsol):
        blockv = bb[:, ich * ns: ich * ns + m] @ a[ipsol[ich]: ipsol[ich + 1], :]
        assert np.allclose(v[ich * ns:(ich + 1) * ns], blockv, rtol=0, atol=1e-12)
        assert np.allclose(w[ich], blockv[-1], rtol=0, atol=1e-12)


def test_channel_weights_restatement():
    """W_OUT's weights (w_out.f90:58-76): sums of squares per channel, SORTA's
    descending order with ties kept in channel order, empty channels weigh 0."""
    rng = np.random.default_rng(11)
    ipsol = np.array([0, 5, 5, 9, 14, 20], np.int32)
    a = rng.standard_normal((20, 20))
    a[:, 3] = 0.1
    a[0:4, 3] = 1.0
    a[4, 3] = 0.0
    a[5:9, 3] = 1.0                     # channels 1 and 3 tie for the largest weight in solution 4
    wt, isol, iprm = O.channel_weights(ipsol, a)
    for s in range(20):
        ref = [sum(a[j, s] * a[j, s] for j in range(ipsol[i], ipsol[i + 1])) for i in range(5)]
        assert list(wt[:, s]) == ref
        order = sorted(range(5), key=lambda i: -ref[i])
        assert ref[iprm[0, s] - 1] == max(ref) and isol[s] == iprm[0, s]
        assert [ref[i - 1] for i in iprm[:, s]] == [ref[i] for i in order]
    assert wt[1].max() == 0.0
    assert wt[0, 3] == wt[2, 3] == max(wt[:, 3])
    assert isol[3] == 1 and list(iprm[:2, 3]) == [1, 3]
