"""Edge cases of the assembly and the eigensolve against the oracle: a partial wave
with no coefficient records, one channel, multipoles without records (ragged
coefficient sets), an exchange group with more records than the factored kernel
stages in shared memory at once, and ks at both ends of the compiled range (3..16).

Tolerances as in test_gpu_assemble (1e-12 per block) and test_gpu_diag (1e-11
relative to the spectral radius)."""
import numpy as np
import pytest

from bsr_b200 import workload as W
from oracle import oracle as O
from tests.gpu_helpers import to_np
from tests.test_gpu_assemble import TOL_H, block_errors, gpu_assemble, oracle_assemble

pytestmark = pytest.mark.gpu
TOL_E = 1e-11


def _records(rows):
    """Coefficient arrays from (k, type, ich, jch, a, b, c) rows, sorted by (k, type, ich, jch)."""
    rows = sorted(rows, key=lambda r: r[:4])
    cols = list(zip(*rows)) if rows else [[]] * 7
    out = {n: np.array(cols[q], dtype=np.int32) for q, n in enumerate(("k", "type", "ich", "jch", "a", "b"))}
    out["c"] = np.array(cols[6], dtype=np.float64)
    return out


def _assemble_matches(pw):
    ob, ref = oracle_assemble(pw, want_acf=False)
    gb, ctx, out = gpu_assemble(pw, want=False)
    errs = block_errors(to_np(out["hcc"]), ref["hcc"])
    assert errs.max() < TOL_H, errs.max()
    return gb, ctx, out


def test_no_coefficient_records():
    """Only the one-electron part: diagonal blocks as the oracle's, off-diagonal blocks zero."""
    pw = W.partial_wave("config1", seed=21)
    pw["coefs"] = _records([])
    gb, ctx, out = _assemble_matches(pw)
    h = to_np(out["hcc"])
    nch = pw["nch"]
    for i in range(2, nch + 1):
        for j in range(1, i):
            assert not h[:, :, i * (i - 1) // 2 + j - 1].any()


def test_one_channel_assembly_and_eigensolve():
    import bsr_b200 as bsr
    pw = W.partial_wave("config1", seed=22, nch=1)
    gb, ctx, out = _assemble_matches(pw)
    H = bsr.assemble(ctx, gb, pw["z"], pw["lch"], pw["ech"], pw["P"], pw["kmax"], pw["coefs"], want_s=True)
    res = bsr.diag_hd(ctx, gb, pw["lch"], H["hcc"], want_vectors=True)
    ref = O.diag_hd(to_np(H["hcc"]).transpose(2, 0, 1), to_np(H["scc"]).transpose(2, 0, 1), pw["lch"], gb.ns,
                    gb.ks, want_vectors=True)
    assert res["khm"] == ref["khm"]
    ev = to_np(res["eval"])
    assert np.max(np.abs(ev - ref["eval"])) / np.max(np.abs(ref["eval"])) < TOL_E


def test_multipoles_without_records():
    """Records at k = 0 and k = kmax only, for a few channel pairs: the multipoles in
    between have no group at all."""
    pw = W.partial_wave("config1", seed=23)
    rng = np.random.default_rng(23)
    rows = []
    for k in (0, pw["kmax"]):
        for (i, j) in ((1, 1), (3, 2), (8, 1)):
            for ty in (0, 1):
                for _ in range(5):
                    a, b = sorted(rng.integers(0, pw["norb"], 2))
                    rows.append((k, ty, i, j, int(a), int(b), float(rng.uniform(-1, 1))))
    pw["coefs"] = _records(rows)
    _assemble_matches(pw)


def test_exchange_group_larger_than_a_record_chunk():
    """At ks = 8 the factored exchange kernel stages up to 2256 records of a chunk in
    shared memory; a group of 2600 records is read from global memory instead, between
    staged chunks before and after it."""
    pw = W.partial_wave("config1", seed=24)
    rng = np.random.default_rng(24)
    norb = pw["norb"]
    rows = []
    for (i, j) in ((2, 1), (3, 3), (5, 4), (7, 2), (8, 8)):
        for ty in (0, 1):
            n = 2600 if (i, j, ty) == (5, 4, 1) else 4
            for q in range(n):
                a, b = (q % norb, (q // norb) % norb) if n > 4 else sorted(rng.integers(0, norb, 2))
                rows.append((2, ty, i, j, int(a), int(b), float(rng.uniform(-1, 1)) / (30.0 if n > 4 else 1.0)))
    pw["coefs"] = _records(rows)
    _assemble_matches(pw)


@pytest.mark.parametrize("ks,ns", [(3, 40), (12, 70)])
def test_assembly_at_the_ends_of_ks(ks, ns):
    pw = W.partial_wave("config1", seed=25, ks=ks, ns=ns, kmax=2, nch=4)
    _assemble_matches(pw)


def test_ks_16_tables_and_assembly():
    """ks = 16, the largest the library is compiled for: mrk_cell bit for bit, and the
    assembly through the per-group gather exchange kernel (the factored kernel is
    compiled up to ks = 12) to the oracle's blocks."""
    import bsr_b200 as bsr
    pw = W.partial_wave("config1", seed=26, ks=16, ns=48, kmax=1, nch=2)
    gb = bsr.define_spline(pw["t"], pw["ks"])
    ob = O.Basis(pw["ks"], pw["t"])
    for k in (0, 1):
        assert np.array_equal(to_np(bsr.mrk_cell(gb, k)), ob.mrk_cell(k))
    _assemble_matches(pw)
