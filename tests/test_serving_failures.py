"""Host logic of the serving loop's failure handling and memory accounting
(CPU; the device objects are replaced by fakes that count the bytes they
hold).

* a request whose footprint is above the budget is rejected, one whose
  set-up raises is failed, one whose residual becomes NaN/Inf is reported
  diverged -- each as its own Result -- and every other request is served;
* the bytes held at any moment (admitted cases, finished cases not yet
  freed, cases set up ahead of admission) never exceed the budget;
* everything set up is freed by the end, failures included.
"""
import numpy as np
import pytest


class Ledger:
    def __init__(self):
        self.held = 0
        self.peak = 0
        self.live = set()

    def take(self, obj, n):
        self.held += n
        self.peak = max(self.peak, self.held)
        self.live.add(id(obj))

    def give(self, obj, n):
        if id(obj) in self.live:
            self.live.discard(id(obj))
            self.held -= n


def fakes(serve, ledger, footprint, poisoned=(), failing=(), iters_to_converge=3):
    """Fake DeviceMesh / Case / Batch; a case's bytes are its footprint,
    taken when it is created and given back when it is closed."""
    A = serve.A

    class FakeDeviceMesh:
        def __init__(self, ctx, mesh):
            self.mesh = mesh

        def close(self):
            pass

    class FakeCase:
        def __init__(self, dm, cfg):
            self.rid = dm.mesh.rid
            if self.rid in failing:
                raise RuntimeError(f"set-up of request {self.rid} failed")
            self.nbytes = footprint(dm.mesh)
            ledger.take(self, self.nbytes)
            self.iters = 0

        def set_field(self, *a):
            pass

        def get_field(self, *a):
            return np.zeros(1)

        def set_graph_mode(self, on=True):
            pass

        def simple_iterate(self, n):
            if self.rid in poisoned:
                raise serve.XcalError(A._abi.XCAL_ERR_DIVERGED, "residual is NaN/Inf")
            k = max(0, min(n, iters_to_converge - self.iters))
            self.iters += k
            return np.full((k, 4), 1e-9), True

        def close(self):
            ledger.give(self, self.nbytes)

    class FakeBatch:
        def __init__(self, ctx, max_cases, budget):
            self.cases, self.budget, self.max_cases = [], budget, max_cases
            self.charge = {}
            self.last_diverged = []

        def add(self, case, charge=0):
            if len(self.cases) >= self.max_cases or sum(self.charge.values()) + charge > self.budget:
                return False
            self.cases.append(case)
            self.charge[id(case)] = charge
            return True

        def remove(self, case):
            self.cases.remove(case)
            self.charge.pop(id(case))

        def simple_iterate(self):
            n = len(self.cases)
            res = np.full((n, 4), 1e-3)
            conv = np.zeros(n, dtype=bool)
            self.last_diverged = []
            for k, c in enumerate(list(self.cases)):
                if c.rid in poisoned:
                    res[k] = np.nan
                    self.last_diverged.append(c)
                    self.remove(c)
                    continue
                c.iters += 1
                conv[k] = c.iters >= iters_to_converge
            return res, conv

        def timings(self):
            return {}

        def close(self):
            pass

    return FakeDeviceMesh, FakeCase, FakeBatch


@pytest.fixture
def serve(x):
    from importlib import import_module
    return import_module(x.__name__ + ".serve")


def _stream(serve, n):
    reqs = serve.make_requests(n, seed=11, n_min=300, n_max=3000, rate=100.0)
    for r in reqs:
        r.build()
        r.mesh.rid = r.rid  # lets the fakes know which request a mesh is
    return reqs


@pytest.mark.parametrize("threads", [0, 2])
def test_failures_stay_with_their_request(serve, monkeypatch, threads):
    reqs = _stream(serve, 10)
    sizes = {r.rid: 1000 + 100 * r.rid for r in reqs}
    big = reqs[2].rid
    sizes[big] = 10 ** 9                     # above any budget below
    ledger = Ledger()
    DM, CS, BT = fakes(serve, ledger, lambda m: sizes[m.rid], poisoned={reqs[5].rid}, failing={reqs[7].rid})
    monkeypatch.setattr(serve.A, "DeviceMesh", DM)
    monkeypatch.setattr(serve.A, "Case", CS)
    monkeypatch.setattr(serve.A, "Batch", BT)
    monkeypatch.setattr(serve.Server, "footprint", lambda self, req: sizes[req.rid])
    budget = 5000
    srv = serve.Server(ctx=None, budget_bytes=budget, max_cases=4, precision="mixed", max_iters=50,
                       build_threads=threads, prepare_ahead=3, free_every=2)
    res = srv.run(reqs, realtime=False)
    st = {r.rid: r.status for r in res}
    assert len(res) == len(reqs)
    assert st[big] == "rejected"
    assert st[reqs[5].rid] == "diverged"
    assert st[reqs[7].rid] == "failed" and "set-up" in [r for r in res if r.rid == reqs[7].rid][0].error
    assert all(st[r.rid] == "converged" for r in reqs if r.rid not in (big, reqs[5].rid, reqs[7].rid))
    assert ledger.peak <= budget, ledger.peak
    assert ledger.held == 0 and not ledger.live
    s = serve.summarize(res, srv.wall)
    assert s["status_counts"] == {"converged": 7, "max_iters": 0, "diverged": 1, "rejected": 1, "failed": 1}


def test_reservations_bound_set_up_ahead(serve, monkeypatch):
    """Cases set up ahead of admission count against the budget: with room
    for two cases at a time, no more than two ever hold memory."""
    reqs = _stream(serve, 8)
    ledger = Ledger()
    DM, CS, BT = fakes(serve, ledger, lambda m: 1000, iters_to_converge=5)
    monkeypatch.setattr(serve.A, "DeviceMesh", DM)
    monkeypatch.setattr(serve.A, "Case", CS)
    monkeypatch.setattr(serve.A, "Batch", BT)
    monkeypatch.setattr(serve.Server, "footprint", lambda self, req: 1000)
    srv = serve.Server(ctx=None, budget_bytes=2000, max_cases=8, precision="mixed", max_iters=50,
                       build_threads=2, prepare_ahead=6, free_every=16, solo_tail=False)
    res = srv.run(reqs, realtime=False)
    assert [r.status for r in res] == ["converged"] * 8
    assert ledger.peak <= 2000, ledger.peak
    assert ledger.held == 0
