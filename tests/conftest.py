import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "test_bs_golden.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libbsrgpu.so")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except Exception:
        have_gpu = False
    if have_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def test_bs(golden):
    """The reference's TEST_BS setup: knot.dat grid (grid_type 0) and the t.f90
    hydrogenic orbitals (Z=2 for 1s, Z=1 for n>1) that produced int_out."""
    from oracle import oracle as O
    kn = golden["knot"]
    grid = O.mkgrid(0, kn["ks"], kn["z"], kn["h"], kn["hmax"], kn["rmax"])
    B = O.Basis(kn["ks"], grid["t"], grid["ml"], grid["me"], grid["h"])
    orbs = {}
    for n in range(1, 6):
        for l in range(n):
            orbs["%d%s" % (n, "spdfg"[l])] = B.bhwf(n, l, kn["z"] if n == 1 else 1.0)
    return {"grid": grid, "basis": B, "orbs": orbs, "knot": kn}


def rel_err(a, b):
    """max|a-b| / max|b| (normwise relative error)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))
