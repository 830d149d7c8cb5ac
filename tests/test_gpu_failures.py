"""Failure detection and isolation on the GPU, made on the host (no device
fault, no trap, no endless wait):

* a case whose initial velocity is poisoned with NaN diverges inside a batch:
  the batch retires it (status XCAL_ERR_DIVERGED in its row) and the other
  cases' results are the same bit for bit as in a batch without it;
* the same in a serving stream: the poisoned request ends as "diverged",
  every other request's result is unchanged bit for bit;
* the bounded grid-barrier wait gives up by its poll limit when a block
  never arrives (one block waiting for a second that is not launched), sets
  its error flag, and the context keeps running work;
* a Krylov solve that stops at itmax is reported (the reference warns,
  Solve_1_api.jl:302) and the run carries on.
"""
import numpy as np
import pytest

from test_gpu_batch import SPECS, _mk

pytestmark = pytest.mark.gpu


def _poison(case, x, n):
    U = np.zeros((3, n))
    U[0, n // 2] = np.nan
    case.set_field(x._abi.FIELD_U, U)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_retires_diverged_case(x, ctx, prec):
    runs = []
    for with_bad in (False, True):
        batch = x.api.Batch(ctx, 8, 1 << 34)
        good = [_mk(x, ctx, kind, n, seed, prec, nu) for kind, n, seed, nu in SPECS[:3]]
        bad = _mk(x, ctx, "channel", 9, 5, prec, 1e-3)
        for c, _ in good[:2]:
            assert batch.add(c)
        if with_bad:
            _poison(bad[0], x, bad[0].mesh.n_cells)
            assert batch.add(bad[0])
        assert batch.add(good[2][0])
        diverged = []
        for _ in range(4):
            res, conv = batch.simple_iterate()
            diverged += batch.last_diverged
        if with_bad:
            assert diverged == [bad[0]] and bad[0] not in batch.cases
            assert batch.info()[0] == 3
        runs.append([(c.get_field(x._abi.FIELD_U), c.get_field(x._abi.FIELD_P)) for c, _ in good])
        batch.close()
    for (U0, p0), (U1, p1) in zip(runs[0], runs[1]):
        assert np.array_equal(U0, U1) and np.array_equal(p0, p1)


def test_serving_poisoned_request(x, ctx):
    from importlib import import_module
    serve = import_module(x.__name__ + ".serve")

    class Poisoned(serve.Request):
        def config(self, precision, max_iters, convergence):
            model, config, pref = super().config(precision, max_iters, convergence)
            model.momentum.U[0, model.momentum.U.shape[1] // 3] = np.nan
            return model, config, pref

    def stream(poison):
        reqs = serve.make_requests(5, seed=3, n_min=300, n_max=3000, rate=50.0)
        if poison:
            r = reqs[2]
            reqs[2] = Poisoned(r.rid, r.kind, r.dims, r.aspect, r.Re, r.arrival)
        srv = serve.Server(ctx, budget_bytes=1 << 33, max_cases=8, precision="mixed", max_iters=40,
                           convergence=1e-12, keep_fields=True)
        return {r.rid: r for r in srv.run(reqs, realtime=False)}

    clean, mixed = stream(False), stream(True)
    assert mixed[2].status == "diverged" and not mixed[2].converged
    for rid, r in clean.items():
        if rid == 2:
            continue
        m = mixed[rid]
        assert m.status == r.status and m.iterations == r.iterations == 40
        assert np.array_equal(m.U, r.U) and np.array_equal(m.p, r.p)


def test_bounded_wait_gives_up(x, ctx):
    import ctypes as C
    from importlib import import_module
    L = import_module(x.__name__ + "._lib").lib()
    gave, flag, after = C.c_int32(-1), C.c_int32(-1), C.c_int32(-1)
    code = L.xcal_check_bounded_wait(ctx.h, 1 << 15, C.byref(gave), C.byref(flag), C.byref(after))
    assert code == 0, L.xcal_last_error(ctx.h)
    assert gave.value == 1 and flag.value == 1 and after.value == 1
    # the context still solves
    c, keep = _mk(x, ctx, "cavity", 12, 1, "fp64", 0.01)
    res, _ = c.simple_iterate(2)
    assert np.all(np.isfinite(res))
    assert L.xcal_check_bounded_wait(ctx.h, 0, None, None, None) == x._abi.XCAL_ERR_INVALID


def test_itmax_is_reported(x, ctx):
    mesh = x.build_mesh3(x.channel_polymesh(16, 8, 8, seed=3))
    model, config = x.cases.channel_case(mesh, iterations=3)
    config.solvers["p"].itmax = 2
    config.solvers["p"].rtol = 1e-12
    cfg, keep = x.build_config(model, config)
    dm = x.DeviceMesh(ctx, mesh)
    c = x.Case(dm, cfg)
    c.set_field(x._abi.FIELD_U, model.momentum.U)
    c.set_field(x._abi.FIELD_P, model.momentum.p)
    c.simple_iterate(3)
    rep = c.solve_report()
    assert rep["status"][3] == 2 and rep["iterations"][3] == 2
    assert rep["itmax_hits"] >= 3
    c.close()
    dm.close()
    model, config = x.cases.channel_case(mesh, iterations=2)
    config.solvers["p"].itmax = 2
    config.solvers["p"].rtol = 1e-12
    with pytest.warns(RuntimeWarning, match="Maximum number of iterations reached"):
        x.run_(model, config)
