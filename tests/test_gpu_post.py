"""The steps either side of the eigensolve on the GPU: BS_ORTH (bs_orth.f90:2-92)
against the oracle's restatement, rsol_out (rsol_out.f90:20-36) against the
oracle and against the generalized eigenproblem itself, and the h.nnn/rsol.nnn
files written from the device results."""
import numpy as np
import pytest

from bsr_b200 import workload as W
from oracle import oracle as O
from tests.gpu_helpers import to_np

pytestmark = pytest.mark.gpu


def _lists(nch, norb):
    return [[i % norb, (i + 3) % norb] if i % 2 == 0 else ([] if i % 3 else [i % norb]) for i in range(nch)]


@pytest.fixture(scope="module")
def solved():
    import bsr_b200 as bsr
    pw = W.partial_wave("config1")
    gb = bsr.define_spline(pw["t"], pw["ks"])
    ctx = bsr.Context()
    H = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"], want_s=True,
                     want_acf=True)
    res = bsr.diag_hd(ctx, gb, pw["lch"], H["hcc"], want_vectors=True, want_bb=True)
    return pw, gb, ctx, H, res


def test_bs_orth_matches_oracle():
    import bsr_b200 as bsr
    pw = W.partial_wave("config1")
    gb = bsr.define_spline(pw["t"], pw["ks"])
    ctx = bsr.Context()
    H = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"])
    h0 = to_np(H["hcc"]).transpose(2, 0, 1)
    lists = _lists(pw["nch"], pw["norb"])
    bsr.bs_orth(ctx, gb, pw["P"], lists, H["hcc"])
    got = to_np(H["hcc"]).transpose(2, 0, 1)
    ob = O.Basis(pw["ks"], pw["t"])
    want = O.bs_orth(ob, pw["P"], lists, h0)
    assert np.max(np.abs(got - want)) / np.max(np.abs(want)) < 1e-12
    # a block whose channels have no condition on either side is untouched
    free = [i for i, l in enumerate(lists) if not l]
    i, j = max(free), min(free)
    assert np.array_equal(got[i * (i + 1) // 2 + j], h0[i * (i + 1) // 2 + j])


def test_bs_orth_no_conditions_is_identity():
    import bsr_b200 as bsr
    pw = W.partial_wave("config1")
    gb = bsr.define_spline(pw["t"], pw["ks"])
    ctx = bsr.Context()
    H = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"])
    h0 = H["hcc"].clone()
    bsr.bs_orth(ctx, gb, pw["P"], [[] for _ in range(pw["nch"])], H["hcc"])
    import torch
    torch.cuda.synchronize()
    assert torch.equal(h0, H["hcc"])


def test_bs_orth_rejects_bad_orbital():
    import bsr_b200 as bsr
    from bsr_b200._lib import BsrgError
    pw = W.partial_wave("config1")
    gb = bsr.define_spline(pw["t"], pw["ks"])
    ctx = bsr.Context()
    H = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"])
    with pytest.raises(BsrgError, match="out of range"):
        bsr.bs_orth(ctx, gb, pw["P"], [[pw["norb"]]] + [[] for _ in range(pw["nch"] - 1)], H["hcc"])


def test_rsol_out_matches_oracle(solved):
    import bsr_b200 as bsr
    pw, gb, ctx, H, res = solved
    ns, nch = gb.ns, pw["nch"]
    ipsol = res["ipsol"]
    assert ipsol[-1] == res["khm"]
    v, w = bsr.rsol_out(ctx, ns, ipsol, res["bb"], res["vectors"])
    _, w2 = bsr.rsol_out(ctx, ns, ipsol, res["bb"], res["vectors"], want_v=False)
    vr, wr = O.rsol(ns, nch, ipsol, to_np(res["bb"]), to_np(res["vectors"]))
    assert np.max(np.abs(to_np(v) - vr)) < 1e-12 * max(1.0, np.max(np.abs(vr)))
    assert np.max(np.abs(to_np(w) - wr)) < 1e-12 * max(1.0, np.max(np.abs(wr)))
    assert np.max(np.abs(to_np(w2) - wr)) < 1e-12 * max(1.0, np.max(np.abs(wr)))


def test_rsol_solutions_solve_h_c_e_s_c(solved):
    """The B-spline-basis solutions satisfy H v = E S v of the assembled blocks."""
    import bsr_b200 as bsr
    pw, gb, ctx, H, res = solved
    ns, nch = gb.ns, pw["nch"]
    v, w = bsr.rsol_out(ctx, ns, res["ipsol"], res["bb"], res["vectors"])
    v = to_np(v)
    ev = to_np(res["eval"])
    hcc = to_np(H["hcc"]).transpose(2, 0, 1)
    scc = to_np(H["scc"]).transpose(2, 0, 1)
    n = nch * ns
    Hf = np.zeros((n, n))
    Sf = np.zeros((n, n))
    for i in range(nch):
        for j in range(i + 1):
            b = i * (i + 1) // 2 + j
            Hf[i * ns:(i + 1) * ns, j * ns:(j + 1) * ns] = hcc[b]
            Hf[j * ns:(j + 1) * ns, i * ns:(i + 1) * ns] = hcc[b].T
            Sf[i * ns:(i + 1) * ns, j * ns:(j + 1) * ns] = scc[b]
            Sf[j * ns:(j + 1) * ns, i * ns:(i + 1) * ns] = scc[b].T
    r = Hf @ v - (Sf @ v) * ev[None, :]
    hn = np.linalg.norm(Hf, 2)
    # the solutions live in the kept channel solutions (|w| >= Egap): the
    # residual vanishes on that space, BB^T (H v - E S v) = 0
    bb = to_np(res["bb"])
    ipsol = res["ipsol"]
    BB = np.zeros((n, res["khm"]))
    for i in range(nch):
        m = ipsol[i + 1] - ipsol[i]
        BB[i * ns:(i + 1) * ns, ipsol[i]:ipsol[i + 1]] = bb[:, i * ns:i * ns + m]
    assert np.max(np.abs(BB.T @ r)) / hn < 1e-10
    # S-normalisation: v^T S v = 1
    assert np.max(np.abs(np.einsum("ij,ij->j", v, Sf @ v) - 1.0)) < 1e-10


def test_h_and_rsol_files(solved, tmp_path):
    import bsr_b200 as bsr
    from bsr_b200 import hout_io
    pw, gb, ctx, H, res = solved
    ns, nch = gb.ns, pw["nch"]
    v, w = bsr.rsol_out(ctx, ns, res["ipsol"], res["bb"], res["vectors"])
    ev, w, v = to_np(res["eval"]), to_np(w), to_np(v)
    acf = to_np(H["acf"])
    p = tmp_path / "h.001"
    hout_io.write_h(p, nelc=2, nz=int(pw["z"]), lamax=pw["kmax"], ra=pw["t"][-1], etarg=[-1.0, -0.5],
                    ltarg=[0, 1], istarg=[1, 3], iptarg=[1, -1], lrgl=1, nspn=1, npty=0, lch=pw["lch"],
                    iptar=[1 + (i % 2) for i in range(nch)], cf=acf, eval_=ev, wmat=w)
    h = hout_io.read_h(p)
    assert h["nchan"] == nch and h["mnp2"] == len(ev) and h["lamax"] == pw["kmax"]
    assert np.array_equal(h["eval"], ev[::-1]) and np.array_equal(h["wmat"], w[:, ::-1])
    assert np.array_equal(h["cf"], acf[:, :, 1:])
    assert list(h["nconat"]) == [4, 4]
    q = tmp_path / "rsol.001"
    hout_io.write_rsol(q, ns, nch, ev, v)
    r = hout_io.read_rsol(q)
    assert r["nhm"] == nch * ns and np.array_equal(r["v"], v) and np.array_equal(r["eval"], ev)


def test_channel_weights_matches_oracle(solved):
    """W_OUT's weights, dominant channel and SORTA order from the device
    eigenvectors equal the oracle's bit for bit."""
    import bsr_b200 as bsr
    pw, gb, ctx, H, res = solved
    wt, isol, iprm = bsr.channel_weights(ctx, res["ipsol"], res["vectors"])
    wr, ir, pr = O.channel_weights(res["ipsol"], to_np(res["vectors"]))
    assert np.array_equal(to_np(wt), wr)
    assert np.array_equal(to_np(isol), ir) and np.array_equal(to_np(iprm), pr)
    # the weights of an S-orthonormal solution in the orthonormal channel basis sum to 1
    assert np.max(np.abs(wr.sum(axis=0) - 1.0)) < 1e-12


def test_channel_weights_chunks_and_many_channels():
    """khm above one shared-memory chunk (2048 rows), more channels than threads
    per block, empty channels: still the oracle's values bit for bit."""
    import torch

    import bsr_b200 as bsr
    rng = np.random.default_rng(21)
    nch = 150
    sizes = rng.integers(0, 36, nch)
    sizes[[3, 77, 149]] = 0
    ipsol = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    khm = int(ipsol[-1])
    assert khm > 2048
    a = np.asfortranarray(rng.standard_normal((khm, khm)))
    ctx = bsr.Context()
    wt, isol, iprm = bsr.channel_weights(ctx, ipsol, torch.from_numpy(a).cuda().t().contiguous().t())
    wr, ir, pr = O.channel_weights(ipsol, a)
    assert np.array_equal(to_np(wt), wr)
    assert np.array_equal(to_np(isol), ir) and np.array_equal(to_np(iprm), pr)
    _, isol2, none = bsr.channel_weights(ctx, ipsol, torch.from_numpy(a).cuda().t().contiguous().t(),
                                         want_iprm=False)
    assert none is None and np.array_equal(to_np(isol2), ir)


def test_channel_weights_rejects_bad_offsets():
    import torch

    import bsr_b200 as bsr
    ctx = bsr.Context()
    a = torch.zeros((6, 6), dtype=torch.float64, device="cuda")
    with pytest.raises(bsr.BsrgError):
        bsr.channel_weights(ctx, np.array([0, 4, 3, 6], np.int32), a)


def test_bound_and_w_files_from_device(solved, tmp_path):
    """b_out.f90's bound.nnn from the device solutions: the states below Emax,
    their energies and B-spline vectors read back to the precision of the format."""
    import bsr_b200 as bsr
    from bsr_b200 import hout_io
    pw, gb, ctx, H, res = solved
    ns, nch = gb.ns, pw["nch"]
    v, _ = bsr.rsol_out(ctx, ns, res["ipsol"], res["bb"], res["vectors"])
    wt, isol, iprm = bsr.channel_weights(ctx, res["ipsol"], res["vectors"])
    ev, v, isol, wt, iprm = to_np(res["eval"]), to_np(v), to_np(isol), to_np(wt), to_np(iprm)
    iptar = [1 + (i % 2) for i in range(nch)]
    etarg = [float(ev[0]) + 0.5, float(ev[0]) + 1.0]
    emax = float(ev[len(ev) // 3])
    pb, pu = tmp_path / "bound.001", tmp_path / "ubound.001"
    nb = hout_io.write_bound(pb, pu, ns, ev, v, isol, iptar, etarg, nz=int(pw["z"]), nelc=int(pw["z"]) - 1, lpar=1,
                             ispar=1, ipar=1, emax=emax, msol=0, iub=-1)
    keep, eb, effn, _ = hout_io.bound_states(ev, isol, iptar, etarg, int(pw["z"]), int(pw["z"]) - 1, emax, 0)
    r = hout_io.read_bound(pb)
    assert nb == r["nbound"] == int(keep.sum()) == int(np.sum(ev <= emax))
    for st, i in zip(r["states"], np.nonzero(keep)[0]):
        assert abs(st["eval"] - ev[i]) <= 5e-10 * abs(ev[i])
        scale = np.max(np.abs(v[:, i]))
        assert np.max(np.abs(st["v"] - v[:, i])) <= 5e-8 * scale
    pw_ = tmp_path / "w.001"
    hout_io.write_w(pw_, wt, isol, ev, np.zeros_like(iprm), [""] * len(ev), iprm)
    w = hout_io.read_w(pw_)
    assert np.array_equal(w["wt"], wt) and np.array_equal(w["isol"], isol)
