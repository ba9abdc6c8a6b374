"""The generalized branch of diag_hd (channel-channel overlap blocks: DPOTRF,
DSYGST, DSYEV, DTRSM of diag_hd.f90:268-334) on the GPU against the oracle's
restatement of the same steps (scipy LAPACK dpotrf/dsygst/dsyev/solve_triangular).

The overlap blocks between channels are seeded multiples (|eps_ij| <= 0.05) of the
B-spline overlap added to the assembled S of config 1.  Refined eigenvalues (Rayleigh
quotients of the standard problem L^-1 A L^-T on both sides) are compared per
eigenvalue; the rounding of forming L^-1 A L^-T differs between the two
reductions, so the bar is 1e-10 (floor 1e-3) rather than the block-diagonal
branch's 1e-11.  The eigenvectors must satisfy A x = E C x and x^T C x = 1."""
import numpy as np
import pytest

from bsr_b200 import workload as W
from oracle import oracle as O
from tests.gpu_helpers import to_np

pytestmark = pytest.mark.gpu


def _perturbed_overlap(scc, ns, ks, eps=0.05, seed=11):
    """Channel-channel overlap blocks eps_ij S (S the B-spline overlap, eps_ij in [-eps, eps]):
    in the S-orthonormal channel bases they become eps_ij bb_i^T S bb_j, of norm <= eps, so the
    transformed overlap C = I + ... stays positive definite."""
    rng = np.random.default_rng(seed)
    nb = scc.shape[0]
    nch = int(round((np.sqrt(8 * nb + 1) - 1) / 2))
    out = scc.copy()
    for i in range(nch):
        for j in range(i):
            out[i * (i + 1) // 2 + j] += rng.uniform(-eps, eps) * scc[0]
    return out


@pytest.mark.parametrize("refine", [True, False])
def test_generalized_config1(refine):
    import bsr_b200 as bsr
    pw = W.partial_wave("config1")
    gb = bsr.define_spline(pw["t"], pw["ks"])
    ctx = bsr.Context()
    ctx.set_refine(refine)
    H = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"], want_s=True)
    hcc = to_np(H["hcc"]).transpose(2, 0, 1)
    scc = _perturbed_overlap(to_np(H["scc"]).transpose(2, 0, 1), gb.ns, gb.ks)
    scc_dev = bsr.as_fortran(np.ascontiguousarray(scc.transpose(1, 2, 0)))
    res = bsr.diag_hd(ctx, gb, pw["lch"], H["hcc"], want_vectors=True, scc=scc_dev)
    ref = O.diag_hd(hcc, scc, pw["lch"], gb.ns, gb.ks, want_vectors=True, refine=refine)
    assert ref["generalized"]
    assert res["khm"] == ref["khm"]
    ev = to_np(res["eval"])
    if refine:
        rel = np.abs(ev - ref["eval"]) / np.maximum(np.abs(ref["eval"]), 1e-3)
        print("generalized config1 refined: per-eigenvalue max rel %.2e" % rel.max())
        assert np.max(rel) <= 1e-10
    else:
        assert np.max(np.abs(ev - ref["eval"])) / np.max(np.abs(ref["eval"])) < 1e-11
    # x in the channel basis: A x = E C x, x^T C x = I, with A and C rebuilt by the oracle in the
    # GPU's channel-basis signs
    X = to_np(res["vectors"])
    khm, ip = res["khm"], ref["ipsol"]
    bbg = to_np(bsr.diag_hd(ctx, gb, pw["lch"], H["hcc"], want_vectors=False, want_bb=True, scc=scc_dev)["bb"])
    nch, ns = pw["nch"], gb.ns
    sg = np.ones(khm)
    for ic in range(nch):
        for q in range(ip[ic + 1] - ip[ic]):
            sg[ip[ic] + q] = np.sign(bbg[:, ic * ns + q] @ ref["bb"][ic][:, q])
    Xs = X * sg[:, None]
    A = np.zeros((khm, khm))
    for i in range(nch):
        for j in range(i + 1):
            A[ip[i]:ip[i + 1], ip[j]:ip[j + 1]] = ref["bb"][i].T @ hcc[i * (i + 1) // 2 + j] @ ref["bb"][j]
    A = np.tril(A) + np.tril(A, -1).T
    C = ref["c"]
    # C here is the oracle's, built in the oracle's channel bases; the GPU's channel eigenvectors
    # differ from them by ~eps ||C_ch|| / gap (1e-10 measured), which bounds this check
    assert np.max(np.abs(Xs.T @ C @ Xs - np.eye(khm))) < 1e-8
    assert np.max(np.abs(A @ Xs - C @ Xs * ev[None, :])) < 1e-11 * np.max(np.abs(A))


def test_generalized_not_positive_definite():
    """An overlap whose channel coupling makes C indefinite stops with the reference's error."""
    import bsr_b200 as bsr
    pw = W.partial_wave("config1")
    gb = bsr.define_spline(pw["t"], pw["ks"])
    ctx = bsr.Context()
    H = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"], want_s=True)
    scc = to_np(H["scc"]).transpose(2, 0, 1).copy()
    scc[1] = 2.0 * scc[0]          # block (2,1) = 2 S: C has a 2x2 block [[I, 2I], [2I, I]] -- indefinite
    scc_dev = bsr.as_fortran(np.ascontiguousarray(scc.transpose(1, 2, 0)))
    with pytest.raises(bsr.BsrgError, match="Cholesky"):
        bsr.diag_hd(ctx, gb, pw["lch"], H["hcc"], want_vectors=True, scc=scc_dev)
