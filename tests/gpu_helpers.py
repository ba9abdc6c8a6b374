"""Shared set-up for the GPU parity tests (CUDA path through the C ABI vs the oracle)."""
import numpy as np

from bsr_b200 import workload as W


def to_np(x):
    """A Fortran-layout CUDA tensor as a Fortran-ordered numpy array."""
    import torch
    torch.cuda.synchronize()
    return np.asfortranarray(x.detach().cpu().numpy())


def grids():
    """(name, ks, t, ml, me, h): the TEST_BS grid (me > 0, scaling-law branch) and
    the semi-exponential benchmark grids (me = 0)."""
    from oracle import oracle as O
    g = O.mkgrid(0, 8, 2.0, 0.125, 160.0, 160.0)
    out = [("test_bs", 8, g["t"], g["ml"], g["me"], g["h"])]
    for name in ("config1", "config2"):
        cfg = W.CONFIGS[name]
        t, _ = W.knot_grid(cfg["ks"], cfg["ns"], cfg["rmin"], cfg["rmax"])
        out.append((name, cfg["ks"], t, 0, 0, 0.0))
    return out


def sub_problem(pw, chans):
    """The coefficients of pw restricted to channels `chans` (1-based, ascending),
    relabelled 1..len(chans): blocks of the sub-problem equal those of the full one."""
    c = pw["coefs"]
    pos = {ch: q + 1 for q, ch in enumerate(chans)}
    keep = np.array([(i in pos and j in pos) for i, j in zip(c["ich"], c["jch"])])
    sub = {k: v[keep].copy() for k, v in c.items()}
    sub["ich"] = np.array([pos[i] for i in sub["ich"]], dtype=np.int32)
    sub["jch"] = np.array([pos[j] for j in sub["jch"]], dtype=np.int32)
    order = np.lexsort((sub["b"], sub["a"], sub["jch"], sub["ich"], sub["type"], sub["k"]))
    sub = {k: v[order] for k, v in sub.items()}
    return {**pw, "nch": len(chans), "lch": pw["lch"][[ch - 1 for ch in chans]],
            "ech": pw["ech"][[ch - 1 for ch in chans]], "coefs": sub}
