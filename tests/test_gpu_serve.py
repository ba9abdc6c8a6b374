"""Resident R^k tables, batching and serving on the GPU (bsr_b200/serve.py).

A request's result must not depend on what else runs: the same symmetry solved
alone and inside a concurrent mix gives identical eigenvalues, and assembly with
the resident tables equals assembly that builds the tables per call."""
import numpy as np
import pytest

from bsr_b200 import workload as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch():
    b = W.symmetry_batch("config4", nsym=64)
    small = [s for s in b["symmetries"] if s["nch"] <= 14][:6]
    assert len(small) >= 4
    return b, small


def test_tables_equal_per_call(batch):
    import torch
    from bsr_b200 import core
    b, small = batch
    basis = core.define_spline(b["t"], b["ks"])
    ctx = core.Context()
    s = small[0]
    h0 = core.assemble(ctx, basis, b["z"], s["lch"], s["ech"], b["P"], b["kmax"], s["coefs"])["hcc"].clone()
    tabs = core.Tables(ctx, basis, b["kmax"])
    assert tabs.nbytes() > 0
    ctx.use_tables(tabs)
    h1 = core.assemble(ctx, basis, b["z"], s["lch"], s["ech"], b["P"], b["kmax"], s["coefs"])["hcc"]
    torch.cuda.synchronize()
    assert torch.equal(h0, h1)
    ctx.use_tables(None)
    tabs.free()


def test_tables_reject_other_basis(batch):
    from bsr_b200 import core
    b, small = batch
    basis = core.define_spline(b["t"], b["ks"])
    other = core.define_spline(b["t"], b["ks"])
    ctx = core.Context()
    tabs = core.Tables(ctx, basis, b["kmax"] - 1)
    ctx.use_tables(tabs)
    s = small[0]
    # tables of another basis, or too few multipoles: assemble builds its own (still correct)
    h_other = core.assemble(ctx, other, b["z"], s["lch"], s["ech"], b["P"], b["kmax"], s["coefs"])["hcc"].clone()
    ctx.use_tables(None)
    h_ref = core.assemble(ctx, basis, b["z"], s["lch"], s["ech"], b["P"], b["kmax"], s["coefs"])["hcc"]
    import torch
    torch.cuda.synchronize()
    assert torch.equal(h_other, h_ref)
    tabs.free()


def test_alone_equals_mix(batch):
    from bsr_b200 import serve
    b, small = batch
    srv = serve.PartialWaveServer(b["t"], b["ks"], b["z"], b["P"], b["kmax"], n_streams=1)
    try:
        alone = [serve.run_stream(srv, [s], [0.0], want_vectors=False)[0].wait(60) for s in small]
    finally:
        srv.close()
    srv = serve.PartialWaveServer(b["t"], b["ks"], b["z"], b["P"], b["kmax"], n_streams=3)
    try:
        order = list(range(len(small)))[::-1] + list(range(len(small)))
        reqs = serve.run_stream(srv, [small[q] for q in order], [0.0] * len(order), want_vectors=False)
        mixed = [r.wait(60) for r in reqs]
        st = srv.stats(reqs)
        assert st["solves"] == len(order) and st["p99_s"] >= st["p50_s"] > 0
    finally:
        srv.close()
    for q, res in zip(order, mixed):
        assert res["khm"] == alone[q]["khm"]
        assert np.array_equal(res["eval"], alone[q]["eval"]), "symmetry %d differs in a mix" % q


def test_matches_single_solve(batch):
    """Served eigenvalues equal the plain assemble + diag_hd path."""
    import torch
    from bsr_b200 import core, serve
    b, small = batch
    s = small[1]
    basis = core.define_spline(b["t"], b["ks"])
    ctx = core.Context()
    H = core.assemble(ctx, basis, b["z"], s["lch"], s["ech"], b["P"], b["kmax"], s["coefs"])
    ref = core.diag_hd(ctx, basis, s["lch"], H["hcc"], want_vectors=False)["eval"].cpu().numpy()
    srv = serve.PartialWaveServer(b["t"], b["ks"], b["z"], b["P"], b["kmax"], n_streams=2)
    try:
        got = srv.submit(s, want_vectors=False).wait(60)
    finally:
        srv.close()
    torch.cuda.synchronize()
    assert np.array_equal(got["eval"], ref)


def test_budget_rejects(batch):
    from bsr_b200 import serve
    b, small = batch
    srv = serve.PartialWaveServer(b["t"], b["ks"], b["z"], b["P"], b["kmax"], n_streams=1,
                                  hbm_budget_bytes=1 << 20)
    try:
        r = srv.submit(small[0])
        with pytest.raises(RuntimeError, match="HBM budget"):
            r.wait(5)
    finally:
        srv.close()


def test_alone_equals_mix_with_vectors(batch):
    """With eigenvectors the workers of a multi-stream server use the library's two-stage
    eigensolver; a request's eigenvalues are still bitwise those of the same request alone
    on a one-stream server using that eigensolver."""
    from bsr_b200 import serve
    b, small = batch
    srv = serve.PartialWaveServer(b["t"], b["ks"], b["z"], b["P"], b["kmax"], n_streams=1, eigensolver="own")
    try:
        alone = [serve.run_stream(srv, [s], [0.0])[0].wait(120) for s in small]
    finally:
        srv.close()
    srv = serve.PartialWaveServer(b["t"], b["ks"], b["z"], b["P"], b["kmax"], n_streams=3)
    assert srv.eigensolver == "own"
    try:
        order = list(range(len(small)))[::-1] + list(range(len(small)))
        mixed = [r.wait(120) for r in serve.run_stream(srv, [small[q] for q in order], [0.0] * len(order))]
    finally:
        srv.close()
    for q, res in zip(order, mixed):
        assert res["khm"] == alone[q]["khm"]
        assert np.array_equal(res["eval"], alone[q]["eval"]), "symmetry %d differs in a mix" % q


def test_mixed_form_alone_equals_mix(batch):
    """The mixed-precision form served: a request's eigenvalues alone and in a concurrent
    mix are bitwise the same (the digit products sum in integers, so their order does not
    matter), and within 1e-10 per eigenvalue (floor 1e-3) of the FP64 form of the same
    request."""
    from bsr_b200 import serve
    b, small = batch
    srv = serve.PartialWaveServer(b["t"], b["ks"], b["z"], b["P"], b["kmax"], n_streams=1, eigensolver="own")
    try:
        fp64 = [serve.run_stream(srv, [s], [0.0])[0].wait(120) for s in small]
    finally:
        srv.close()
    srv = serve.PartialWaveServer(b["t"], b["ks"], b["z"], b["P"], b["kmax"], n_streams=1, eigensolver="own",
                                  mixed=True)
    try:
        alone = [serve.run_stream(srv, [s], [0.0])[0].wait(120) for s in small]
    finally:
        srv.close()
    srv = serve.PartialWaveServer(b["t"], b["ks"], b["z"], b["P"], b["kmax"], n_streams=3, mixed=True)
    assert srv.eigensolver == "own" and srv.mixed
    try:
        order = list(range(len(small)))[::-1] + list(range(len(small)))
        mix = [r.wait(120) for r in serve.run_stream(srv, [small[q] for q in order], [0.0] * len(order))]
    finally:
        srv.close()
    for q, res in zip(order, mix):
        assert res["khm"] == alone[q]["khm"]
        assert np.array_equal(res["eval"], alone[q]["eval"]), "symmetry %d differs in a mix" % q
    for a, f in zip(alone, fp64):
        rel = np.abs(a["eval"] - f["eval"]) / np.maximum(np.abs(f["eval"]), 1e-3)
        assert rel.max() <= 1e-10


def test_warm_then_serve(batch):
    """PartialWaveServer.warm solves one symmetry on every worker outside the served
    results; what is served afterwards is unchanged."""
    from bsr_b200 import serve
    b, small = batch
    srv = serve.PartialWaveServer(b["t"], b["ks"], b["z"], b["P"], b["kmax"], n_streams=3)
    try:
        srv.warm(max(small, key=lambda s: s["nch"]))
        assert srv.done == []
        got = serve.run_stream(srv, small[:2], [0.0, 0.0])
        res = [r.wait(120) for r in got]
        assert len(srv.done) == 2
    finally:
        srv.close()
    srv = serve.PartialWaveServer(b["t"], b["ks"], b["z"], b["P"], b["kmax"], n_streams=1, eigensolver="own")
    try:
        alone = [serve.run_stream(srv, [s], [0.0])[0].wait(120) for s in small[:2]]
    finally:
        srv.close()
    for a, r in zip(alone, res):
        assert np.array_equal(a["eval"], r["eval"])
