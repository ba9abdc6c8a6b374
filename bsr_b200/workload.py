"""Seeded synthetic partial-wave workloads (host logic, numpy only).

The reference's own inputs for this path come from its angular pipeline
(bsr_prep/bsr_conf/bsr_breit writing int_bnk) and from target orbitals; those
stages are outside this path.  These generators stand in for them with the
shapes the partial-wave benchmarks use:

  knots     exponential from r_min (t_{i+1} = t_i e^{0.25 s}) until the spacing
            reaches 0.25 s, then linear to Rmax; ks-fold knots at 0 and Rmax.
            The scale s is chosen (bisection on the interval count) so that
            the grid has exactly ns splines.  No scaling-law shortcut (me = 0).
  orbitals  B-spline coefficients ~ N(0,1), normalised to <P|S|P> = 1.
  channels  l_ch = ch mod lmod, target energies ~ U[-1, 0].
  angular   one Bernoulli(p) draw per (k, structure, channel pair ich >= jch,
            orbital pair a <= b) candidate, value ~ U[-1, 1]; records sorted
            by (k, structure, ich, jch, a, b) as State_res buckets them.
"""
import math

import numpy as np

# the partial-wave configurations of the benchmark suite
CONFIGS = {
    "config1": dict(ks=8, ns=60, rmin=1e-3, rmax=20.0, kmax=4, norb=10, nch=8, lmod=5, z=10.0, p=0.05, seed=1),
    "config2": dict(ks=10, ns=200, rmin=1e-3, rmax=40.0, kmax=8, norb=30, nch=40, lmod=9, z=18.0, p=0.02, seed=2),
    "config4": dict(ks=8, ns=150, rmin=1e-3, rmax=30.0, kmax=6, norb=20, nch=None, lmod=7, z=10.0, p=0.03, seed=4,
                    nsym=64, nch_lo=4, nch_hi=60),
    # serving: the config4 basis and orbitals, a Poisson request stream with 4..80 channels
    "config5": dict(ks=8, ns=150, rmin=1e-3, rmax=30.0, kmax=6, norb=20, nch=None, lmod=7, z=10.0, p=0.03, seed=4,
                    nsym=64, nch_lo=4, nch_hi=80, sym_seed=5, rate_per_s=50.0),
}


def _knots_for_scale(ks, rmin, rmax, s, step=0.25):
    lam, dlin = step * s, step * s
    ex = [rmin]
    while True:
        nxt = ex[-1] * math.exp(lam)
        if nxt - ex[-1] >= dlin or nxt >= rmax:
            break
        ex.append(nxt)
    te = ex[-1]
    nlin = max(1, int(round((rmax - te) / dlin)))
    lin = [te + (rmax - te) * q / nlin for q in range(1, nlin + 1)]
    lin[-1] = rmax
    interior = ex + lin                      # distinct knots after 0, ending at rmax
    return [0.0] * ks + interior[:-1] + [rmax] * ks


def knot_grid(ks, ns, rmin, rmax):
    """Semi-exponential knot sequence with exactly ns splines.  Returns (t, s)."""
    nv_target = ns - ks + 1

    def nv_of(s):
        return len(_knots_for_scale(ks, rmin, rmax, s)) - 2 * ks + 1

    lo, hi = 1e-3, 1e3          # nv decreases with s
    if not (nv_of(lo) >= nv_target >= nv_of(hi)):
        raise ValueError("cannot reach ns=%d" % ns)
    for _ in range(200):
        mid = math.sqrt(lo * hi)
        if nv_of(mid) > nv_target:
            lo = mid
        else:
            hi = mid
    # [hi, right end of the plateau] all give nv_target: take the plateau's middle
    a = hi
    b = hi
    while nv_of(b * 1.001) == nv_target:
        b *= 1.001
    s = math.sqrt(a * b)
    t = np.array(_knots_for_scale(ks, rmin, rmax, s))
    assert len(t) == ns + ks
    return t, s


def overlap_matrix(t, ks):
    """Full <B_i|B_j> by Gauss-Legendre quadrature (for normalising orbitals)."""
    from scipy.interpolate import BSpline

    ns = len(t) - ks
    x, w = np.polynomial.legendre.leggauss(ks)
    tl, tr = t[ks - 1: ns], t[ks: ns + 1]
    pts = ((tr - tl)[:, None] * (x[None, :] + 1) / 2 + tl[:, None]).ravel()
    wts = ((tr - tl)[:, None] * w[None, :] / 2).ravel()
    B = BSpline.design_matrix(pts, t, ks - 1).toarray()
    return B.T @ (wts[:, None] * B)


def orbitals(rng, t, ks, norb):
    ns = len(t) - ks
    S = overlap_matrix(t, ks)
    P = rng.standard_normal((ns, norb))
    for a in range(norb):
        P[:, a] /= math.sqrt(P[:, a] @ S @ P[:, a])
    return np.asfortranarray(P)


def coefficients(rng, nch, norb, kmax, p):
    """Angular coefficient records sorted by (k, type, ich, jch, a, b)."""
    chp = [(i, j) for i in range(1, nch + 1) for j in range(1, i + 1)]
    orp = [(a, b) for a in range(norb) for b in range(a, norb)]
    shape = (kmax + 1, 2, len(chp), len(orp))
    mask = rng.random(shape) < p
    k, ty, cp, op = np.nonzero(mask)
    vals = rng.uniform(-1.0, 1.0, size=len(k))
    chp_a = np.array(chp, dtype=np.int32)
    orp_a = np.array(orp, dtype=np.int32)
    return {
        "k": k.astype(np.int32), "type": ty.astype(np.int32),
        "ich": chp_a[cp, 0].copy(), "jch": chp_a[cp, 1].copy(),
        "a": orp_a[op, 0].copy(), "b": orp_a[op, 1].copy(), "c": vals,
    }


def partial_wave(name="config1", seed=None, nch=None, **over):
    """One partial wave of the named configuration (dict of numpy inputs)."""
    cfg = dict(CONFIGS[name])
    cfg.update(over)
    if seed is None:
        seed = cfg["seed"]
    if nch is None:
        nch = cfg["nch"]
    rng = np.random.default_rng(seed)
    t, s = knot_grid(cfg["ks"], cfg["ns"], cfg["rmin"], cfg["rmax"])
    P = orbitals(rng, t, cfg["ks"], cfg["norb"])
    lch = np.array([ch % cfg["lmod"] for ch in range(nch)], dtype=np.int32)
    ech = rng.uniform(-1.0, 0.0, size=nch)
    coefs = coefficients(rng, nch, cfg["norb"], cfg["kmax"], cfg["p"])
    return {
        "name": name, "seed": seed, "ks": cfg["ks"], "ns": cfg["ns"], "t": t, "knot_scale": s,
        "z": cfg["z"], "kmax": cfg["kmax"], "nch": nch, "norb": cfg["norb"], "lch": lch, "ech": ech,
        "P": P, "coefs": coefs,
    }


def symmetry_batch(name="config4", seed=None, nsym=None):
    """Many partial waves sharing one basis and orbital set (batched workload)."""
    cfg = CONFIGS[name]
    seed = cfg["seed"] if seed is None else seed
    nsym = cfg["nsym"] if nsym is None else nsym
    rng = np.random.default_rng(seed)
    t, s = knot_grid(cfg["ks"], cfg["ns"], cfg["rmin"], cfg["rmax"])
    P = orbitals(rng, t, cfg["ks"], cfg["norb"])
    if "sym_seed" in cfg:                   # shares the basis and orbitals of the seed, own symmetries
        rng = np.random.default_rng(cfg["sym_seed"] + (seed - cfg["seed"]))
    lo, hi = math.log(cfg["nch_lo"]), math.log(cfg["nch_hi"])
    out = []
    for q in range(nsym):
        nch = int(math.floor(math.exp(rng.uniform(lo, hi))))
        lch = np.array([ch % cfg["lmod"] for ch in range(nch)], dtype=np.int32)
        ech = rng.uniform(-1.0, 0.0, size=nch)
        coefs = coefficients(rng, nch, cfg["norb"], cfg["kmax"], cfg["p"])
        out.append({"nch": nch, "lch": lch, "ech": ech, "coefs": coefs})
    return {"name": name, "seed": seed, "ks": cfg["ks"], "ns": cfg["ns"], "t": t, "knot_scale": s,
            "z": cfg["z"], "kmax": cfg["kmax"], "norb": cfg["norb"], "P": P, "symmetries": out}


def request_stream(name="config5", seed=None, nreq=None):
    """Serving workload: symmetries of the config5 distribution with Poisson arrival
    offsets (s) of the configured mean rate.  Returns (batch, arrivals)."""
    cfg = CONFIGS[name]
    b = symmetry_batch(name, seed=seed, nsym=nreq)
    rng = np.random.default_rng((cfg["sym_seed"] if "sym_seed" in cfg else cfg["seed"]) + 7919)
    arrivals = np.cumsum(rng.exponential(1.0 / cfg["rate_per_s"], size=len(b["symmetries"])))
    return b, arrivals
