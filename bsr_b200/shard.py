"""Partial-wave sharding across GPUs (one process per GPU).

Partial-wave symmetries are independent: they share only the B-spline basis
and the orbitals, and a solve needs no data from another symmetry.  The
reference distributes work inside one symmetry over MPI ranks
(src/bsr/BSR_MAT3_MPI: channel blocks dealt round-robin, mod_intmat_mpi.f90:60-66;
src/bsr/BSR_HDB3: ScaLAPACK).  At the sizes here one symmetry fits one B200,
so the B200 layout deals whole symmetries to ranks instead:

  plan_shards   longest-processing-time-first bin packing of symmetries onto
                ranks by a cost model (the dense eigensolve dominates, ~khm^3),
                subject to each rank's HBM budget;
  run_sharded   every rank solves its own symmetries; the only communication is
                the final gather of results to rank 0 (host objects over the
                process group), outside the data path.

A solve that raises is reported as data ({"error": ...}) in the gather instead
of leaving the other ranks waiting; a rank that disappears surfaces as the
process group's timeout error on the others.
"""
import math


def symmetry_dims(nch, ns, lch, ks):
    """(khm upper bound, H bytes, dense bytes) of one symmetry."""
    nch, ns, ks = int(nch), int(ns), int(ks)
    khm = nch * ns - sum(min(int(l), ks - 2) + 1 for l in lch)
    h_bytes = nch * (nch + 1) // 2 * ns * ns * 8
    dense_bytes = 3 * khm * khm * 8          # A, eigenvectors, eigensolver workspace
    return khm, h_bytes, dense_bytes


def solve_cost(nch, ns, lch, ks, kmax=8):
    """Relative cost of one symmetry: dense eigensolve ~ khm^3 plus assembly ~ groups x ns^2 ks^2."""
    khm, _, _ = symmetry_dims(nch, ns, lch, ks)
    pairs = nch * (nch + 1) // 2
    return 9.0 * khm ** 3 + 2.0 * pairs * (kmax + 1) * ns * ns * (2 * ks - 1) ** 2


def plan_shards(symmetries, n_ranks, hbm_budget_bytes, ns, ks, kmax=8):
    """Assign symmetry indices to ranks.

    symmetries: list of dicts with "nch" and "lch".  Returns a list (per rank)
    of symmetry indices, each rank's list in ascending index order.  Raises
    ValueError if a symmetry does not fit a rank's HBM budget at all.  The plan
    is deterministic (ties broken by index)."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    items = []
    for q, s in enumerate(symmetries):
        khm, hb, db = symmetry_dims(s["nch"], ns, s["lch"], ks)
        mem = hb + db
        if mem > hbm_budget_bytes:
            raise ValueError("symmetry %d needs %.2f GB, above the per-rank budget of %.2f GB"
                             % (q, mem / 1e9, hbm_budget_bytes / 1e9))
        items.append((solve_cost(s["nch"], ns, s["lch"], ks, kmax), mem, q))
    items.sort(key=lambda x: (-x[0], x[2]))
    load = [0.0] * n_ranks
    plan = [[] for _ in range(n_ranks)]
    for cost, mem, q in items:
        # symmetries on a rank run one after another, so a rank's peak memory is
        # its largest symmetry; every symmetry already fits, any rank can take it
        r = min(range(n_ranks), key=lambda i: (load[i], i))
        plan[r].append(q)
        load[r] += cost
    return [sorted(p) for p in plan]


def imbalance(plan, symmetries, ns, ks, kmax=8):
    """max rank load / mean rank load of a plan (1.0 = perfect balance)."""
    loads = [sum(solve_cost(symmetries[q]["nch"], ns, symmetries[q]["lch"], ks, kmax) for q in p) for p in plan]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def run_sharded(symmetries, solve_fn, plan, group=None):
    """Solve this rank's share of `symmetries` and gather everything on rank 0.

    solve_fn(index, symmetry) -> result (any picklable object).  Returns, on
    rank 0, the list of results in symmetry order (a failed solve appears as
    {"error": message}); other ranks return None."""
    import torch.distributed as dist

    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    if len(plan) != world:
        raise ValueError("plan has %d ranks, process group has %d" % (len(plan), world))
    mine = {}
    for q in plan[rank]:
        try:
            mine[q] = solve_fn(q, symmetries[q])
        except Exception as ex:          # reported as data: the other ranks must not wait on us
            mine[q] = {"error": "%s: %s" % (type(ex).__name__, ex)}
    if world == 1:
        return [mine[q] for q in range(len(symmetries))]
    gathered = [None] * world if rank == 0 else None
    # dst is a global rank: the group's rank 0 may not be global rank 0
    dst = dist.get_global_rank(group, 0) if group is not None else 0
    dist.gather_object(mine, gathered, dst=dst, group=group)
    if rank != 0:
        return None
    out = [None] * len(symmetries)
    for part in gathered:
        for q, v in part.items():
            out[q] = v
    missing = [q for q, v in enumerate(out) if v is None]
    if missing:
        raise RuntimeError("symmetries %s were not solved by any rank" % missing)
    return out
