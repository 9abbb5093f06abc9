"""Host logic of the served form (mnmgdatalog_b200/serve.py) on CPU, with a
fake session standing in for the GPU one: arrival-order admission, the HBM
budget, continuous batching (requests join while others run) and latency
accounting. The GPU parity of served results is in test_serve_gpu.py."""
import time

import numpy as np

from mnmgdatalog_b200 import serve


class FakeResult:
    def __init__(self, rows, iterations):
        self.rows = rows
        self.output_tuples = len(rows)
        self.iterations = iterations


class FakeSession:
    """Instance i needs (rows % 4) + 1 iterations; its result is the sorted
    input. Holds 1 KiB per active input row."""

    def __init__(self, log):
        self.log = log
        self.inst = {}
        self.active = {}
        self.done = []
        self.closed = False

    def admit(self, edges):
        i = len(self.inst)
        self.inst[i] = edges
        self.log.append(("admit", i, len(self.active)))
        if len(edges) == 0:
            self.done.append(i)
        else:
            self.active[i] = len(edges) % 4 + 1
        return i

    def admit_many(self, edge_sets):
        return [self.admit(e) for e in edge_sets]

    def step(self):
        time.sleep(0.001)  # an iteration takes device time
        for i in list(self.active):
            self.active[i] -= 1
            if self.active[i] == 0:
                del self.active[i]
                self.done.append(i)
        return len(self.active)

    def poll(self):
        d, self.done = self.done, []
        return d

    def result(self, i, output="host", out=None):
        e = self.inst[i]
        return FakeResult(np.sort(e, axis=0), len(e) % 4 + 1)

    def release(self, i):
        self.inst[i] = None

    def memory(self):
        return 1024 * sum(len(self.inst[i]) for i in self.active), len(self.active)

    def close(self):
        self.closed = True


def _server(log, **kw):
    backend = {p: (lambda: FakeSession(log)) for p in serve.PROGRAMS}
    return serve.Server(backend=backend, **kw)


def _requests(n, seed=0, spacing=0.0):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        m = int(rng.integers(0, 40))
        out.append(serve.Request(i, serve.PROGRAMS[i % 3], rng.integers(0, 100, (m, 2)).astype(np.int32),
                                 arrival=i * spacing))
    return out


def test_all_requests_complete_with_their_own_results():
    log = []
    srv = _server(log)
    reqs = _requests(60)
    st = srv.serve(reqs)
    assert st.requests == 60 and len(srv.finished) == 60
    for r in reqs:
        assert r.done >= r.admitted >= r.arrival >= 0
        assert np.array_equal(r.result.rows, np.sort(r.edges, axis=0))
    assert st.latency_p50 <= st.latency_p95 <= st.latency_p99 <= st.latency_max
    assert st.max_active > 1  # batched: several instances ran together
    srv.close()


def test_continuous_batching_admits_while_others_run():
    log = []
    srv = _server(log)
    reqs = _requests(30, seed=1, spacing=0.002)
    srv.serve(reqs)
    # some request was admitted while another instance of its session was active
    assert any(a == "admit" and running > 0 for a, _, running in log)


def test_budget_limits_concurrency_and_keeps_arrival_order():
    log = []
    # every request estimates to ~1 MiB + rows * row_bytes; a budget below two
    # estimates lets exactly one request run at a time
    srv = _server(log, budget_bytes=(1 << 20) + 10)
    srv.row_bytes = {p: 0.0 for p in serve.PROGRAMS}
    reqs = _requests(25, seed=2)
    st = srv.serve(reqs)
    assert st.max_active <= 1
    assert st.waits_on_budget > 0
    order = sorted(reqs, key=lambda r: r.admitted)
    assert [r.id for r in order] == sorted(r.id for r in reqs)


def test_estimate_grows_with_observed_output():
    log = []
    srv = _server(log)
    srv.row_bytes = {p: 1.0 for p in serve.PROGRAMS}
    reqs = _requests(12, seed=3)
    srv.serve(reqs)
    assert all(srv.row_bytes[p] > 1.0 for p in serve.PROGRAMS)


def test_max_active_cap():
    log = []
    srv = _server(log, max_active=2)
    st = srv.serve(_requests(40, seed=4))
    assert st.max_active <= 2


def test_poisson_arrivals_rate():
    rng = np.random.default_rng(0)
    t = serve.poisson_arrivals(20000, 500.0, rng)
    assert np.all(np.diff(t) > 0)
    assert abs(len(t) / t[-1] - 500.0) < 15.0


def test_percentiles():
    p50, p95, p99, mx = serve.percentiles(list(np.arange(1, 101, dtype=float)))
    assert (p50, mx) == (50.5, 100.0) and 95 <= p95 <= 96 and 99 <= p99 <= 100


def test_concurrent_workers_complete_with_their_own_results():
    log = []
    srv = _server(log, concurrent=True)
    reqs = _requests(90, seed=5, spacing=0.0005)
    st = srv.serve(reqs)
    assert st.requests == 90 and len(srv.finished) == 90
    for r in reqs:
        assert r.done >= r.admitted >= r.arrival >= 0
        assert np.array_equal(r.result.rows, np.sort(r.edges, axis=0))
    assert st.max_active > 1


def test_concurrent_budget_and_order():
    log = []
    srv = _server(log, concurrent=True, budget_bytes=(1 << 20) + 10)
    srv.row_bytes = {p: 0.0 for p in serve.PROGRAMS}
    reqs = _requests(24, seed=6)
    st = srv.serve(reqs)
    assert st.max_active <= 1 and st.waits_on_budget > 0
    order = sorted(reqs, key=lambda r: r.admitted)
    assert [r.id for r in order] == sorted(r.id for r in reqs)


def test_concurrent_worker_error_surfaces():
    import pytest

    class Broken(FakeSession):
        def step(self):
            raise RuntimeError("device lost")

    backend = {p: (lambda: Broken([])) for p in serve.PROGRAMS}
    srv = serve.Server(backend=backend, concurrent=True)
    with pytest.raises(RuntimeError, match="device lost"):
        srv.serve(_requests(6, seed=7))


def test_device_headroom_leaves_room_for_worker_caches(monkeypatch):
    """The server's budget is capped by the device memory free at start less
    every worker context's reuse cache and a margin."""
    import torch
    gib = 1 << 30
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda device=None: (100 * gib, 180 * gib))
    assert serve.device_headroom(0, 3, 4) == (100 - 3 * 4 - 2) * gib
    assert serve.device_headroom(0, 1, 96) == 2 * gib
    assert serve.device_headroom(0, 30, 4) == 0  # never negative
