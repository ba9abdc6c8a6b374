"""bsr_mat channel-block assembly on the GPU against the oracle's restatement of
SUB1 / L_data / I_data Case(6..9) / UPDATE_HX,HL,CF (src/bsr/BSR_MAT3).

Tolerance: 1e-12 relative per block, max|dH| / max|H_block| (FP64)."""
import numpy as np
import pytest

from bsr_b200 import workload as W
from oracle import oracle as O
from tests.gpu_helpers import sub_problem, to_np

pytestmark = pytest.mark.gpu
TOL_H = 1e-12


def oracle_assemble(pw, want_acf=True):
    ob = O.Basis(pw["ks"], pw["t"])
    rkb_all = np.stack([ob.mrk_cell(k) for k in range(pw["kmax"] + 1)], axis=-1)
    return ob, O.assemble(ob, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], np.asfortranarray(rkb_all),
                          pw["coefs"], want_s=True, want_acf=want_acf)


def gpu_assemble(pw, want=True):
    import bsr_b200 as bsr
    gb = bsr.define_spline(pw["t"], pw["ks"])
    ctx = bsr.Context()
    out = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"],
                       want_s=want, want_acf=want)
    return gb, ctx, out


def block_errors(h_gpu, h_ref):
    """h_gpu: (ns, ns, nblk) Fortran numpy; h_ref: (nblk, ns, ns) [row, col]."""
    errs = []
    for b in range(h_ref.shape[0]):
        ref = h_ref[b]
        got = h_gpu[:, :, b]
        den = np.max(np.abs(ref))
        errs.append(np.max(np.abs(got - ref)) / den if den > 0 else np.max(np.abs(got)))
    return np.array(errs)


@pytest.fixture(scope="module")
def config1():
    pw = W.partial_wave("config1")
    ob, ref = oracle_assemble(pw)
    gb, ctx, out = gpu_assemble(pw)
    return pw, ref, {k: to_np(v) for k, v in out.items()}


def test_h_blocks_config1(config1):
    pw, ref, got = config1
    errs = block_errors(got["hcc"], ref["hcc"])
    assert errs.max() < TOL_H, errs.max()


def test_overlap_blocks_config1(config1):
    pw, ref, got = config1
    assert np.array_equal(got["scc"].transpose(2, 0, 1), ref["scc"])


def test_asymptotic_coefficients_config1(config1):
    pw, ref, got = config1
    acf_ref = ref["acf"]                       # (k, ich, jch)
    acf_got = got["acf"].transpose(2, 0, 1)
    den = np.max(np.abs(acf_ref))
    assert np.max(np.abs(acf_got - acf_ref)) / den < 1e-12


def test_diagonal_blocks_symmetric(config1):
    pw, ref, got = config1
    nch = pw["nch"]
    for ich in range(1, nch + 1):
        blk = got["hcc"][:, :, ich * (ich + 1) // 2 - 1]
        assert np.array_equal(blk, blk.T)


def test_linearity_in_coefficients():
    """H(2c) - H(c) = H(c) - H(0): the two-electron part is linear in the angular coefficients."""
    pw = W.partial_wave("config1", seed=5)
    h = []
    for s in (0.0, 1.0, 2.0):
        q = dict(pw)
        q["coefs"] = dict(pw["coefs"])
        q["coefs"]["c"] = pw["coefs"]["c"] * s
        h.append(to_np(gpu_assemble(q, want=False)[2]["hcc"]))
    d1, d2 = h[1] - h[0], h[2] - h[1]
    assert np.max(np.abs(d2 - d1)) <= 1e-12 * np.max(np.abs(h[2]))


def test_bad_coefficient_raises():
    import bsr_b200 as bsr
    pw = W.partial_wave("config1")
    c = {k: v.copy() for k, v in pw["coefs"].items()}
    c["ich"][0] = pw["nch"] + 3
    gb = bsr.define_spline(pw["t"], pw["ks"])
    ctx = bsr.Context()
    with pytest.raises(bsr.BsrgError) as ei:
        bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], c)
    assert "out of range" in str(ei.value)


def test_config2_blocks_via_subproblem():
    """Full-size (ns=200, ks=10, k=0..8) blocks: each block depends only on its
    own coefficients, so a sub-problem on 9 channels drawn at random (seeded)
    solved by the oracle gives 45 exact blocks (36 off-diagonal, 9 diagonal) of
    the 40-channel GPU assembly."""
    pw = W.partial_wave("config2")
    gb, ctx, out = gpu_assemble(pw, want=False)
    h = to_np(out["hcc"])
    chans = sorted(int(x) + 1 for x in np.random.default_rng(2024).choice(pw["nch"], 9, replace=False))
    sub = sub_problem(pw, chans)
    ob, ref = oracle_assemble(sub, want_acf=False)
    nblk = 0
    for si in range(1, len(chans) + 1):
        for sj in range(1, si + 1):
            i, j = chans[si - 1], chans[sj - 1]
            rb = ref["hcc"][si * (si - 1) // 2 + sj - 1]
            gbk = h[:, :, i * (i - 1) // 2 + j - 1]
            err = np.max(np.abs(gbk - rb)) / np.max(np.abs(rb))
            assert err < TOL_H, ((i, j), err)
            nblk += 1
    assert nblk == 45


def test_add_two_electron_is_i_data_alone():
    """bsrg_add_two_electron accumulates exactly the I_data groups: on zeroed blocks
    its off-diagonal blocks equal the full assembly's (which holds no other term there)."""
    import torch

    import bsr_b200 as bsr
    pw = W.partial_wave("config1", seed=6)
    gb, ctx, full = gpu_assemble(pw, want=False)
    nch = pw["nch"]
    h2 = torch.zeros_like(full["hcc"])
    bsr.add_two_electron(ctx, gb, nch, pw["P"], pw["kmax"], pw["coefs"], h2)
    a, b = to_np(h2), to_np(full["hcc"])
    for i in range(2, nch + 1):
        for j in range(1, i):
            q = i * (i - 1) // 2 + j - 1
            assert np.array_equal(a[:, :, q], b[:, :, q]), (i, j)


@pytest.mark.parametrize("gather", [False, True])
def test_exchange_paths_match_oracle(monkeypatch, gather):
    """Both exchange kernels -- the factored one (default, norb <= 32) and the
    per-group gather one -- give the oracle's blocks to 1e-12."""
    if gather:
        monkeypatch.setenv("BSRG_EXCHANGE_GATHER", "1")
    pw = W.partial_wave("config1", seed=12)
    ob, ref = oracle_assemble(pw, want_acf=False)
    gb, ctx, out = gpu_assemble(pw, want=False)
    errs = block_errors(to_np(out["hcc"]), ref["hcc"])
    assert errs.max() < TOL_H, errs.max()


@pytest.mark.parametrize("simt", [False, True])
def test_direct_paths_match_oracle(monkeypatch, simt):
    """Both direct contractions -- the reshaped table times the group densities by
    cuBLAS DGEMM (default) and the register-tiled SIMT kernel (BSRG_DIRECT_SIMT) --
    give the oracle's blocks to 1e-12, and agree with each other to 1e-13."""
    pw = W.partial_wave("config1", seed=13)
    ob, ref = oracle_assemble(pw, want_acf=False)
    if simt:
        monkeypatch.setenv("BSRG_DIRECT_SIMT", "1")
    gb, ctx, out = gpu_assemble(pw, want=False)
    errs = block_errors(to_np(out["hcc"]), ref["hcc"])
    assert errs.max() < TOL_H, errs.max()
