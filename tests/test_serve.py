"""Serving / batching host logic (bsr_b200/serve.py) without a GPU: the admission
queue keeps the HBM budget, starts requests in arrival order, never starves."""
import threading
import time

import numpy as np

from bsr_b200 import serve


class _R:
    def __init__(self, rid, nbytes):
        self.rid, self.nbytes = rid, nbytes


def _drain(q, n_workers, hold_s, log):
    def work():
        while True:
            r = q.take()
            if r is None:
                return
            log.append(("start", r.rid, q.in_flight))
            time.sleep(hold_s)
            q.release(r)
    ths = [threading.Thread(target=work) for _ in range(n_workers)]
    for t in ths:
        t.start()
    return ths


def test_budget_respected_and_fifo():
    q = serve.AdmissionQueue(100)
    sizes = [40, 40, 40, 90, 10, 10, 60]
    log = []
    for i, s in enumerate(sizes):
        q.put(_R(i, s))
    ths = _drain(q, 4, 0.02, log)
    time.sleep(0.3)
    q.close()
    for t in ths:
        t.join()
    starts = [rid for kind, rid, _ in log if kind == "start"]
    assert starts == list(range(len(sizes)))              # arrival order
    assert q.peak <= 100 and q.in_flight == 0


def test_oversized_request_runs_alone():
    q = serve.AdmissionQueue(50)
    log = []
    q.put(_R(0, 10))
    q.put(_R(1, 500))                                       # above the budget: admitted only when alone
    ths = _drain(q, 2, 0.02, log)
    time.sleep(0.2)
    q.close()
    for t in ths:
        t.join()
    big = [inflight for kind, rid, inflight in log if rid == 1]
    assert big == [500]


def test_request_bytes_grow_with_channels():
    a = serve.request_bytes(4, 150, [0, 1, 2, 3], 8)
    b = serve.request_bytes(40, 150, [c % 7 for c in range(40)], 8)
    assert b > 50 * a


def test_poisson_arrivals():
    rng = np.random.default_rng(0)
    t = serve.poisson_stream(rng, 50.0, 2000)
    assert np.all(np.diff(t) > 0)
    assert abs(2000 / t[-1] - 50.0) < 5.0


def test_request_bytes_numpy_ints():
    """Channel counts and l values arrive as numpy int32: no 32-bit overflow at 80 channels."""
    lch = np.arange(80, dtype=np.int32) % 7
    nb = serve.request_bytes(np.int32(80), np.int32(150), lch, 8)
    assert isinstance(nb, int) and nb > 3 * 11000 ** 2 * 8


class _FakeServer:
    def __init__(self, n, rate):
        self.n, self.rate, self.done, self.warmed, self.closed = n, rate, [], [], False

    def warm(self, sym, want_vectors=True, timeout=600.0):
        self.warmed.append(sym)

    def stats(self, reqs):
        return {"solves_per_s": self.rate}

    def close(self):
        self.closed = True


def test_autotune_prefers_more_streams_within_margin(monkeypatch):
    """The most streams within 5 % of the best rate win; every candidate's workers are
    warmed first with the sample's largest symmetry; the choice and the measured rates go
    to the cache."""
    made = []

    def fake_run(srv, syms, arrivals, want_vectors=True):
        assert srv.warmed, "timed before the warm-up"
        return list(syms)

    monkeypatch.setattr(serve, "run_stream", fake_run)
    sample = [{"nch": c} for c in (4, 9, 30, 7, 12, 5, 8, 6)]
    for rates, want in (({1: 10.0, 2: 10.3, 4: 9.0}, 2), ({1: 12.5, 2: 11.0, 4: 9.0}, 1),
                        ({1: 10.0, 2: 10.0, 4: 13.0}, 4), ({1: 9.7, 2: 9.9, 4: 9.95}, 4)):
        made.clear()

        def make(n, rates=rates):
            made.append(_FakeServer(n, rates[n]))
            return made[-1]

        cache = {}
        assert serve.autotune_streams(make, sample, candidates=(1, 2, 4), cache=cache, key="k") == want
        assert [s.warmed for s in made] == [[{"nch": 30}]] * 3 and all(s.closed for s in made)
        assert cache["k"] == {"n_streams": want, "solves_per_s": rates}
        assert serve.autotune_streams(make, sample, candidates=(1, 2, 4), cache=cache, key="k") == want
        assert len(made) == 3                   # the cached choice runs nothing


def test_request_bytes_counts_the_library_eigensolver():
    lch = [c % 7 for c in range(40)]
    a = serve.request_bytes(40, 150, lch, 8)
    b = serve.request_bytes(40, 150, lch, 8, own_eig=True)
    khm = 40 * 150 - sum(min(l, 6) + 1 for l in lch)
    assert b - a == int((6.5 * khm * khm + 3000 * khm) * 8)
    # without eigenvectors neither eigensolver workspace nor the refinement is counted
    assert serve.request_bytes(40, 150, lch, 8, want_vectors=False, own_eig=True) == \
        serve.request_bytes(40, 150, lch, 8, want_vectors=False)


def test_request_bytes_counts_the_mixed_form_digits():
    """The mixed-precision form holds the 8-bit digit planes of the refinement's product
    (16 bytes per element of A, rounded up to the product's tiles) and of the direct
    contraction on top of the FP64 form's buffers."""
    lch = [c % 7 for c in range(40)]
    khm = serve.shard.symmetry_dims(40, 150, lch, 8)[0]
    a = serve.request_bytes(40, 150, lch, 8)
    b = serve.request_bytes(40, 150, lch, 8, mixed=True)
    assert b - a >= 16 * khm * khm
    c = serve.request_bytes(40, 150, lch, 8, want_vectors=False, mixed=True)
    assert c - serve.request_bytes(40, 150, lch, 8, want_vectors=False) < 16 * khm * khm
