"""Partial-wave sharding (bsr_b200/shard.py): planning, and the two-rank
gather path on CPU with the gloo backend (world size 2)."""
import os
import socket

import numpy as np
import pytest

from bsr_b200 import shard
from bsr_b200 import workload as W


def _syms(n=24, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        nch = int(np.floor(np.exp(rng.uniform(np.log(4), np.log(60)))))
        out.append({"nch": nch, "lch": [ch % 7 for ch in range(nch)]})
    return out


def test_plan_covers_every_symmetry_once_and_balances():
    syms = _syms()
    plan = shard.plan_shards(syms, 4, 180e9, ns=150, ks=8)
    flat = sorted(q for p in plan for q in p)
    assert flat == list(range(len(syms)))
    assert shard.imbalance(plan, syms, 150, 8) < 1.35
    assert plan == shard.plan_shards(syms, 4, 180e9, ns=150, ks=8)       # deterministic


def test_plan_respects_the_hbm_budget():
    syms = [{"nch": 80, "lch": list(range(80))}]
    with pytest.raises(ValueError, match="budget"):
        shard.plan_shards(syms, 2, 1e9, ns=150, ks=8)


def test_single_rank_runs_without_a_process_group():
    syms = _syms(5)
    plan = shard.plan_shards(syms, 1, 180e9, ns=150, ks=8)
    out = shard.run_sharded(syms, lambda q, s: q * 10, plan)
    assert out == [0, 10, 20, 30, 40]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _solve(q, sym):
    """A stand-in solve on the host: eigenvalues of a small seeded matrix per symmetry."""
    rng = np.random.default_rng(q)
    n = 4 + sym["nch"] % 7
    a = rng.standard_normal((n, n))
    if sym.get("fail"):
        raise RuntimeError("channel diagonalization failed")
    return np.linalg.eigvalsh(a + a.T).tolist()


def _worker(rank, world, port, syms, mode, outq):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=8))
    plan = shard.plan_shards(syms, world, 180e9, ns=150, ks=8)
    try:
        if mode == "vanish" and rank == 1:
            outq.put((rank, "left"))
            return                       # leaves between steps, before the gather
        res = shard.run_sharded(syms, _solve, plan)
        outq.put((rank, res))
    except Exception as ex:
        outq.put((rank, "error: %s" % type(ex).__name__))
    finally:
        if not (mode == "vanish" and rank == 1):
            try:
                dist.destroy_process_group()
            except Exception:
                pass


def _run_two(syms, mode):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, syms, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, v = q.get(timeout=120)
        res[r] = v
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return res


def test_two_ranks_gather_all_results():
    syms = _syms(9, seed=1)
    res = _run_two(syms, "ok")
    ref = [_solve(q, s) for q, s in enumerate(syms)]
    assert res[1] is None
    assert res[0] == ref


def test_failed_solve_is_reported_not_hung():
    syms = _syms(6, seed=2)
    syms[3]["fail"] = True
    res = _run_two(syms, "ok")
    assert res[0][3] == {"error": "RuntimeError: channel diagonalization failed"}
    assert all(isinstance(v, list) for q, v in enumerate(res[0]) if q != 3)


def test_vanished_rank_ends_in_an_error_on_rank0():
    syms = _syms(6, seed=3)
    res = _run_two(syms, "vanish")
    assert res[1] == "left"
    assert isinstance(res[0], str) and res[0].startswith("error")
