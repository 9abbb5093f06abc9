"""Served form on the GPU: every result served in the mix (continuous
batching, Poisson arrivals) equals the plain engine's result for the same
request run alone -- rows, iteration count and per-iteration deltas (all
integer, so the tolerance is zero)."""
import numpy as np
import pytest

from mnmgdatalog_b200 import serve

pytestmark = pytest.mark.gpu


def _check(engine, reqs):
    for r in reqs:
        alone = engine.run(r.program, r.edges)
        got = r.result
        assert got.iterations == alone.iterations, r.id
        assert got.deltas.tolist() == alone.deltas.tolist(), r.id
        assert np.array_equal(got.rows, alone.rows), r.id


@pytest.mark.parametrize("concurrent", [False, True], ids=["one_thread", "worker_per_program"])
def test_served_results_equal_alone(engine, concurrent):
    reqs = serve.mixed_requests(90, lo=40, hi=6000, pool=10, seed=1)
    arr = serve.poisson_arrivals(len(reqs), 600.0, np.random.default_rng(2))
    for r, t in zip(reqs, arr):
        r.arrival = float(t)
    srv = serve.Server(engine, concurrent=concurrent)
    try:
        st = srv.serve(reqs)
    finally:
        srv.close()
    assert st.requests == 90 and len(srv.finished) == 90
    assert st.max_active > 1
    assert all(r.done >= r.arrival for r in reqs)
    _check(engine, reqs)


@pytest.mark.parametrize("concurrent", [False, True], ids=["one_thread", "worker_per_program"])
def test_served_under_tight_budget(engine, concurrent):
    reqs = serve.mixed_requests(24, lo=40, hi=3000, pool=6, seed=3)
    srv = serve.Server(engine, budget_bytes=4 << 20, concurrent=concurrent)  # below the sum of the estimates
    try:
        st = srv.serve(reqs)
    finally:
        srv.close()
    assert st.waits_on_budget > 0
    _check(engine, reqs)


def test_plain_service_matches(engine):
    reqs = serve.mixed_requests(9, lo=40, hi=2000, pool=3, seed=4)
    total, svc, res = serve.serve_plain(engine, reqs)
    assert len(svc) == 9 and total >= sum(svc) * 0.99
    for r, x in zip(reqs, res):
        assert np.array_equal(x.rows, engine.run(r.program, r.edges).rows)
