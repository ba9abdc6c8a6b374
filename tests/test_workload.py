"""Host logic: seeded workloads, knot rule, coefficient records."""
import numpy as np
import pytest

from bsr_b200 import workload as W


@pytest.mark.parametrize("name,ks,ns", [("config1", 8, 60), ("config2", 10, 200), ("config4", 8, 150)])
def test_knot_rule_hits_ns(name, ks, ns):
    cfg = W.CONFIGS[name]
    t, s = W.knot_grid(ks, ns, cfg["rmin"], cfg["rmax"])
    assert len(t) == ns + ks
    assert np.all(t[:ks] == 0.0) and np.all(t[-ks:] == cfg["rmax"])
    inner = t[ks - 1: ns + 1]
    assert np.all(np.diff(inner) > 0)
    assert inner[1] == pytest.approx(cfg["rmin"])
    assert 0.5 < s < 2.5


def test_orbitals_normalised():
    pw = W.partial_wave("config1")
    S = W.overlap_matrix(pw["t"], pw["ks"])
    P = pw["P"]
    assert np.allclose(np.einsum("ia,ij,ja->a", P, S, P), 1.0, atol=1e-12)


def test_coefficients_sorted_and_seeded():
    a = W.partial_wave("config1")
    b = W.partial_wave("config1")
    c = a["coefs"]
    for k in c:
        assert np.array_equal(c[k], b["coefs"][k])
    key = ((c["k"] * 2 + c["type"]) * 10_000 + c["ich"] * 100 + c["jch"]) * 10_000 + c["a"] * 100 + c["b"]
    assert np.all(np.diff(key) > 0)
    assert np.all(c["ich"] >= c["jch"]) and np.all(c["a"] <= c["b"])
    n_cand = 5 * 2 * 36 * 55
    assert 0.03 * n_cand < len(c["c"]) < 0.07 * n_cand
    assert W.partial_wave("config1", seed=99)["coefs"]["c"][0] != c["c"][0]


def test_symmetry_batch_shapes():
    sb = W.symmetry_batch("config4", nsym=6)
    assert len(sb["symmetries"]) == 6
    for s in sb["symmetries"]:
        assert 4 <= s["nch"] <= 60 and len(s["lch"]) == s["nch"]
