"""Host logic of the serving loop (no GPU): the seeded request stream and
the latency summary."""
import numpy as np
import pytest


def _serve(x):
    from importlib import import_module
    return import_module(x.__name__ + ".serve")


def test_request_stream_distribution(x):
    serve = _serve(x)
    reqs = serve.make_requests(400, seed=7, n_min=1e3, n_max=5e5, rate=4.0)
    again = serve.make_requests(400, seed=7, n_min=1e3, n_max=5e5, rate=4.0)
    assert [(r.kind, r.dims, r.arrival) for r in reqs] == [(r.kind, r.dims, r.arrival) for r in again]
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) > 0)
    # Poisson arrivals at 4/s: mean gap 0.25 s
    assert np.mean(np.diff(t)) == pytest.approx(0.25, rel=0.2)
    kinds = [r.kind for r in reqs]
    assert 0.4 < kinds.count("cavity") / len(kinds) < 0.6
    n = np.array([r.n_cells for r in reqs], dtype=float)
    assert n.min() >= 0.5e3 and n.max() <= 1.5 * 5e5
    # log-uniform: the median sits near the geometric mean of the range
    assert np.median(np.log(n)) == pytest.approx(0.5 * (np.log(1e3) + np.log(5e5)), abs=0.6)
    assert all(100.0 <= r.Re <= 2000.0 and 1.0 <= r.aspect <= 4.0 for r in reqs)
    assert all(r.dims[2] == 1 for r in reqs if r.kind == "cavity")


def test_summary_percentiles(x):
    serve = _serve(x)
    res = [serve.Result(i, 1000, arrival=0.0, admitted=0.0, finished=(i + 1) / 100.0, iterations=10,
                        converged=i != 3, residuals=np.zeros(4)) for i in range(100)]
    s = serve.summarize(res, wall=2.0)
    assert s["cases"] == 100 and s["converged"] == 99
    assert s["p50_ms"] == pytest.approx(505.0)
    assert s["p99_ms"] == pytest.approx(990.1)
    assert s["mcell_iters_per_s"] == pytest.approx(100 * 1000 * 10 / 2.0 / 1e6)
