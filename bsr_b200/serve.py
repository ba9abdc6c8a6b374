"""Serving and batching of partial-wave solves on one GPU.

A partial-wave solve (bsr_mat SUB1 + bsr_hd diag_hd for one symmetry) is a
request.  The server keeps everything the requests share on the device -- the
B-spline basis, the orbitals and the R^k tables of every multipole (built
once, bsrg_tables) -- and runs the requests on S worker streams, each with its
own library context:

  admission   a request is started when a worker is free and its HBM estimate
              fits the budget left by the requests in flight (largest-first
              is not used: arrival order is kept, a request that does not fit
              waits at the head of the queue);
  batching    continuous: requests that arrive while others run are admitted
              as soon as a worker and memory free up, so their work overlaps
              on the device;
  results     eigenvalues (host numpy), khm, and the submit/start/done times;
              latency percentiles and solves/s over a window.

The batched form of a symmetry list is the same server fed everything at t=0.
Each request runs the same kernels with the same arguments alone or in a mix,
so its result does not depend on what else is in flight.
"""
import queue
import threading
import time

import numpy as np

from . import shard


class Request:
    __slots__ = ("rid", "sym", "want_vectors", "t_submit", "t_start", "t_done", "result", "error", "event", "nbytes",
                 "barrier")

    def __init__(self, rid, sym, want_vectors):
        self.rid, self.sym, self.want_vectors = rid, sym, want_vectors
        self.t_submit = self.t_start = self.t_done = None
        self.result = self.error = None
        self.event = threading.Event()
        self.nbytes = 0
        self.barrier = None       # warm-up requests: the worker waits here after releasing it

    def wait(self, timeout=None):
        if not self.event.wait(timeout):
            raise TimeoutError("request %d not finished" % self.rid)
        if self.error is not None:
            raise RuntimeError(self.error)
        return self.result

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_submit


OWN_EIG_MIN = 7000      # diag_hd's default crossover to the library's dense eigensolver (rows)


def request_bytes(nch, ns, lch, ks, want_vectors=True, own_eig=False, mixed=False):
    """Device bytes one solve needs beyond the shared state (H blocks, the dense
    problem with vectors and its eigensolver workspace, block-transform buffers;
    with vectors also the eigenvectors and the refinement's copy of A and its
    residuals; with the library's two-stage eigensolver its workspace: the band
    reduction's copy, both stages' reflectors and block factors, the divide and
    conquer's merge buffers, ~6.5 khm^2 + 3000 khm doubles; in the mixed-precision
    form the 8-bit digit planes of the refinement's product, 16 bytes per element of
    A rounded up to the product's tiles, and of the direct contraction)."""
    khm, hb, db = shard.symmetry_dims(nch, ns, lch, ks)
    nch, ns = int(nch), int(ns)
    nb = nch * (nch + 1) // 2
    transform = 2 * nb * ns * ns * 8
    channel = 4 * nch * ns * ns * 8
    own = int((6.5 * khm * khm + 3000 * khm) * 8) if (own_eig and want_vectors) else 0
    digits = 0
    if mixed:
        nk = ns * ks          # the direct contraction: (nk x nk) times (nk x direct groups <= nb)
        digits = 8 * (nk + 128 + nb + 64) * (nk + 32) + (16 * (khm + 128) * (khm + 32) if want_vectors else 0)
    return hb + db + transform + channel + (3 * khm * khm * 8 if want_vectors else 0) + own + digits


class AdmissionQueue:
    """FIFO of requests admitted by an HBM budget (no GPU needed).

    take() blocks until the head request fits the memory left by the requests in
    flight (a request alone is always admitted, so nothing starves) or the
    queue is closed and empty; release() returns a finished request's memory."""

    def __init__(self, budget_bytes):
        self.budget = int(budget_bytes)
        self.in_flight = 0
        self.peak = 0
        self._pending = []
        self._cv = threading.Condition()
        self._closing = False

    def put(self, r):
        with self._cv:
            self._pending.append(r)
            self._cv.notify_all()

    def take(self):
        with self._cv:
            while True:
                if self._pending:
                    head = self._pending[0]
                    if self.in_flight + head.nbytes <= self.budget or self.in_flight == 0:
                        self._pending.pop(0)
                        self.in_flight += head.nbytes
                        self.peak = max(self.peak, self.in_flight)
                        return head
                elif self._closing:
                    return None
                self._cv.wait(timeout=0.05)

    def release(self, r):
        with self._cv:
            self.in_flight -= r.nbytes
            self._cv.notify_all()

    def close(self):
        with self._cv:
            self._closing = True
            self._cv.notify_all()


class PartialWaveServer:
    """Device-resident request loop for partial waves sharing one basis and orbital set."""

    def __init__(self, t, ks, z, P, kmax, n_streams=2, hbm_budget_bytes=None, device=0, eigensolver=None,
                 mixed=False):
        """mixed: every worker solves in the mixed-precision form (Context.set_precision:
        the direct contraction and the refinement's A V from 8-bit digits on the tensor
        cores); FP64 by default.
        eigensolver: diag_hd's dense eigensolver per worker ("auto", "own" or "lib", see
        Context.set_eigensolver).  Default: "own" with more than one stream -- concurrent
        solves overlap with the library's two-stage solver, whose bulge chasing and panel
        factorisations leave most of the GPU to the other streams, where cuSOLVER's
        per-column reduction serialises them (config 4 on a B200: 14.9 solves/s on four
        streams against 9.5 to 14.2 from run to run with cuSOLVER) -- and "auto" with one."""
        import torch

        from . import core
        self.torch, self.core = torch, core
        torch.cuda.set_device(device)
        self.device = device
        self.ks, self.ns, self.z, self.kmax = ks, len(t) - ks, float(z), kmax
        self.eigensolver = eigensolver or ("own" if n_streams > 1 else "auto")
        self.mixed = bool(mixed)
        self.basis = core.define_spline(t, ks)
        self.P = core.as_fortran(P)
        self._setup_ctx = core.Context()
        self.tables = core.Tables(self._setup_ctx, self.basis, kmax)
        torch.cuda.synchronize()
        free, total = torch.cuda.mem_get_info()
        self.budget = int(hbm_budget_bytes if hbm_budget_bytes is not None else 0.8 * free)
        self.queue = AdmissionQueue(self.budget)
        self._lock = threading.Lock()
        self._next_id = 0
        self.done = []
        self.workers = []
        for w in range(n_streams):
            th = threading.Thread(target=self._worker, args=(w,), daemon=True)
            th.start()
            self.workers.append(th)

    # ---- client side ----
    def submit(self, sym, want_vectors=True):
        """sym: dict with nch, lch, ech, coefs.  Returns a Request (wait() for the result)."""
        khm = shard.symmetry_dims(sym["nch"], self.ns, sym["lch"], self.ks)[0]
        own = self.eigensolver == "own" or (self.eigensolver == "auto" and khm >= OWN_EIG_MIN)
        nb = request_bytes(sym["nch"], self.ns, sym["lch"], self.ks, want_vectors, own_eig=own, mixed=self.mixed)
        with self._lock:
            r = Request(self._next_id, sym, want_vectors)
            self._next_id += 1
        r.nbytes = nb
        r.t_submit = time.perf_counter()
        if nb > self.budget:
            r.error = "request needs %.2f GB, above the HBM budget of %.2f GB" % (nb / 1e9, self.budget / 1e9)
            r.t_done = r.t_submit
            r.event.set()
            return r
        self.queue.put(r)
        return r

    def warm(self, sym, want_vectors=True, timeout=600.0):
        """Solve `sym` once on every worker, untimed and outside the served results, so that
        each worker's context has grown its device workspace to that problem's size (a
        workspace that grows during service synchronises the device and stalls every
        stream).  Give it the largest symmetry expected.  A worker that has finished its
        copy waits until every worker has taken one, so each worker solves exactly one."""
        n = len(self.workers)
        barrier = threading.Barrier(n, timeout=timeout)
        reqs = []
        for _ in range(n):
            r = self.submit(sym, want_vectors)
            r.barrier = barrier
            reqs.append(r)
        for r in reqs:
            r.wait(timeout)
        with self._lock:
            self.done = [d for d in self.done if d not in reqs]

    def close(self):
        self.queue.close()
        for th in self.workers:
            th.join()
        self.torch.cuda.synchronize()

    def stats(self, reqs=None):
        reqs = [r for r in (reqs if reqs is not None else self.done) if r.error is None and r.t_done is not None]
        if not reqs:
            return {}
        lat = np.array([r.latency for r in reqs])
        t0 = min(r.t_submit for r in reqs)
        t1 = max(r.t_done for r in reqs)
        return {"solves": len(reqs), "solves_per_s": len(reqs) / (t1 - t0), "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()), "window_s": t1 - t0}

    # ---- worker side ----
    def _release(self, r):
        with self._lock:
            self.done.append(r)
        self.queue.release(r)

    def _worker(self, w):
        torch, core = self.torch, self.core
        torch.cuda.set_device(self.device)
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            ctx = core.Context(stream=stream)
            ctx.use_tables(self.tables)
            ctx.set_eigensolver(self.eigensolver)
            ctx.set_precision(self.mixed)
            while True:
                r = self.queue.take()
                if r is None:
                    break
                r.t_start = time.perf_counter()
                try:
                    s = r.sym
                    H = core.assemble(ctx, self.basis, self.z, s["lch"], s["ech"], self.P, self.kmax, s["coefs"])
                    res = core.diag_hd(ctx, self.basis, s["lch"], H["hcc"], want_vectors=r.want_vectors)
                    ev = res["eval"].cpu().numpy()          # synchronises this worker's stream
                    r.result = {"eval": ev, "khm": res["khm"]}
                    del H, res
                except Exception as ex:
                    r.error = "%s: %s" % (type(ex).__name__, ex)
                r.t_done = time.perf_counter()
                r.event.set()
                self._release(r)
                if r.barrier is not None:
                    # a failed warm-up releases the other workers at once instead of at the timeout
                    try:
                        if r.error is not None:
                            r.barrier.abort()
                        else:
                            r.barrier.wait()
                    except threading.BrokenBarrierError:
                        pass
            ctx.close()


def poisson_stream(rng, rate_per_s, n):
    """Arrival offsets (s) of n requests of a Poisson process."""
    return np.cumsum(rng.exponential(1.0 / rate_per_s, size=n))


def run_stream(server, symmetries, arrivals, want_vectors=True):
    """Submit symmetries at the given offsets (s, from now); wait for all; return requests."""
    t0 = time.perf_counter()
    reqs = []
    for sym, at in zip(symmetries, arrivals):
        delay = t0 + at - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        reqs.append(server.submit(sym, want_vectors))
    for r in reqs:
        r.event.wait()
    return reqs


def autotune_streams(make_server, sample, candidates=(1, 2, 4), cache=None, key=None, margin=0.05):
    """Pick the worker-stream count with the highest solves/s on a sample batch.

    make_server(n_streams) -> PartialWaveServer; sample: list of symmetries.  Each
    candidate server's workers first solve the sample's largest symmetry once
    (PartialWaveServer.warm), so no worker grows its workspace in the timed run.  A short sample's rates are noisy and
    close together, while on a full batch more workers also overlap each other's host
    work (record grouping, uploads, result reads), so the most streams whose rate is
    within `margin` of the best is chosen.  The choice is kept in `cache` (a dict, e.g.
    loaded from JSON) under `key`."""
    if cache is not None and key in cache:
        return cache[key]["n_streams"]
    rates = {}
    for n in candidates:
        srv = make_server(n)
        try:
            srv.warm(max(sample, key=lambda s: s["nch"]))
            reqs = run_stream(srv, sample, [0.0] * len(sample), want_vectors=True)
            rates[n] = srv.stats(reqs)["solves_per_s"]
        finally:
            srv.close()
    top = max(rates.values())
    best = max(n for n in candidates if rates[n] >= top / (1.0 + margin))
    if cache is not None:
        cache[key] = {"n_streams": best, "solves_per_s": rates}
    return best
