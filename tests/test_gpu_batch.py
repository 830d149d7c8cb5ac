"""Batching and serving: a case advanced inside a batch (one batched launch
sequence per Krylov solve over all resident cases) gives the same results,
bit for bit, as the same case advanced alone through xcal_simple_iterate --
FP64 and mixed precision, cavity and channel meshes of uneven size; the
serving loop's results are the same alone and in the mix; admission honours
the device-memory budget; the footprint estimate bounds the allocation."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mk(x, ctx, kind, n, seed, prec, nu):
    A = x.api
    if kind == "cavity":
        mesh = x.build_mesh3(x.cavity_polymesh(n, seed=seed, nx=n + 3, lx=1.3))
        model, config = x.cases.cavity_case(mesh, iterations=50, precision=prec, nu=nu)
        pref = 0.0
    else:
        mesh = x.build_mesh3(x.channel_polymesh(n + 4, n, n - 1, seed=seed, length=2.0))
        model, config = x.cases.channel_case(mesh, iterations=50, precision=prec, nu=nu)
        pref = None
    cfg, keep = x.build_config(model, config, pref=pref)
    dm = A.DeviceMesh(ctx, mesh)
    c = A.Case(dm, cfg)
    # the batch's FP32 inner CG is the canonical form (a case takes it when
    # admitted); a case solved alone in that form is identical bit for bit
    c.set_inner_cg(1)
    c.set_field(x._abi.FIELD_U, model.momentum.U)
    c.set_field(x._abi.FIELD_P, model.momentum.p)
    return c, (dm, keep, cfg)


SPECS = [("cavity", 18, 1, 0.01), ("channel", 10, 2, 2e-3), ("cavity", 31, 3, 1e-3), ("channel", 7, 4, 1e-2)]


@pytest.mark.parametrize("persist", [True, False, 256])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_matches_single(x, ctx, prec, persist):
    """persist: the batch runs its CG solves as one cooperative launch over
    every member (True: widest block form that fits; 256: the narrow form) or
    as the batched two-kernel loop (False); the cases alone use the
    persistent single-case kernel either way."""
    iters = 6
    alone = []
    for kind, n, seed, nu in SPECS:
        c, keep = _mk(x, ctx, kind, n, seed, prec, nu)
        res, _ = c.simple_iterate(iters)
        alone.append((res, c.get_field(x._abi.FIELD_U), c.get_field(x._abi.FIELD_P)))
    batch = x.api.Batch(ctx, 8, 1 << 34)
    members = []
    for kind, n, seed, nu in SPECS:
        c, keep = _mk(x, ctx, kind, n, seed, prec, nu)
        c.set_persistent(persist)
        assert batch.add(c)
        members.append((c, keep))
    hist = []
    for _ in range(iters):
        r, conv = batch.simple_iterate()
        hist.append(r)
    hist = np.stack(hist, axis=1)  # [case, iter, 4]
    for k, (c, keep) in enumerate(members):
        assert np.array_equal(hist[k], alone[k][0]), (k, hist[k], alone[k][0])
        assert np.array_equal(c.get_field(x._abi.FIELD_U), alone[k][1])
        assert np.array_equal(c.get_field(x._abi.FIELD_P), alone[k][2])
    batch.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_cluster_form_matches_single(x, ctx, prec):
    """Cases of 2, 5 and 10 tiles: the batch runs every pressure CG as one
    thread-block cluster per case (16 blocks each, padding blocks without
    rows); alone, each case runs the 1024-thread cooperative form.  Same
    results, bit for bit."""
    specs = [("cavity", 60, 7, 1e-3), ("channel", 20, 8, 2e-3), ("channel", 26, 9, 5e-3)]
    iters = 3
    alone = []
    for kind, n, seed, nu in specs:
        c, keep = _mk(x, ctx, kind, n, seed, prec, nu)
        c.set_persistent(1024)
        res, _ = c.simple_iterate(iters)
        alone.append((res, c.get_field(x._abi.FIELD_U), c.get_field(x._abi.FIELD_P)))
    batch = x.api.Batch(ctx, 4, 1 << 34)
    members = []
    for kind, n, seed, nu in specs:
        c, keep = _mk(x, ctx, kind, n, seed, prec, nu)
        c.set_persistent(2)
        assert batch.add(c)
        members.append((c, keep))
    hist = np.stack([batch.simple_iterate()[0] for _ in range(iters)], axis=1)
    for k, (c, keep) in enumerate(members):
        assert np.array_equal(hist[k], alone[k][0]), (k, hist[k], alone[k][0])
        assert np.array_equal(c.get_field(x._abi.FIELD_U), alone[k][1])
        assert np.array_equal(c.get_field(x._abi.FIELD_P), alone[k][2])
    batch.close()


def test_batch_enter_leave_keeps_results(x, ctx):
    """A case that joins a running batch later and one that leaves early give
    the results they give alone."""
    prec = "mixed"
    ref = []
    for kind, n, seed, nu in SPECS[:3]:
        c, keep = _mk(x, ctx, kind, n, seed, prec, nu)
        res, _ = c.simple_iterate(5)
        ref.append(c.get_field(x._abi.FIELD_P))
    batch = x.api.Batch(ctx, 4, 1 << 34)
    cs = [_mk(x, ctx, kind, n, seed, prec, nu) for kind, n, seed, nu in SPECS[:3]]
    assert batch.add(cs[0][0]) and batch.add(cs[1][0])
    batch.simple_iterate()
    batch.simple_iterate()
    assert batch.add(cs[2][0])          # joins at iteration 3 of the others
    for _ in range(3):
        batch.simple_iterate()
    batch.remove(cs[0][0])              # case 0 has done 5 iterations
    assert np.array_equal(cs[0][0].get_field(x._abi.FIELD_P), ref[0])
    batch.simple_iterate()
    batch.simple_iterate()              # case 2 reaches 5
    assert np.array_equal(cs[2][0].get_field(x._abi.FIELD_P), ref[2])
    batch.close()


def test_batch_budget_and_footprint(x, ctx):
    c1, k1 = _mk(x, ctx, "channel", 12, 1, "mixed", 1e-3)
    cb, mb = c1.footprint()
    est = x.api.footprint_estimate(c1.mesh, "mixed", dilu_U=True, dilu_p=False)
    assert cb + mb <= est <= 1.25 * (cb + mb), (cb, mb, est)
    batch = x.api.Batch(ctx, 4, est + est // 2)
    assert batch.add(c1, est)
    c2, k2 = _mk(x, ctx, "channel", 12, 2, "mixed", 1e-3)
    assert not batch.add(c2, est)        # over budget: refused, nothing changed
    n, used, budget = batch.info()
    assert n == 1 and used == est
    batch.remove(c1)
    assert batch.add(c2, est)
    batch.close()


def test_serving_same_alone_and_in_mix(x, ctx):
    from importlib import import_module
    serve = import_module(x.__name__ + ".serve")
    reqs = serve.make_requests(5, seed=3, n_min=300, n_max=3000, rate=50.0)
    server = serve.Server(ctx, budget_bytes=1 << 33, max_cases=8, precision="mixed", max_iters=40,
                          convergence=1e-12, keep_fields=True)
    mix = server.run(reqs, realtime=False)
    assert len(mix) == 5
    for r in reqs:
        r.mesh = None
    for req in reqs:
        solo = serve.Server(ctx, budget_bytes=1 << 33, max_cases=8, precision="mixed", max_iters=40,
                            convergence=1e-12, keep_fields=True).run([req], realtime=False)[0]
        m = mix[req.rid]
        assert m.iterations == solo.iterations == 40
        assert np.array_equal(m.U, solo.U) and np.array_equal(m.p, solo.p)
    s = serve.summarize(mix, server.wall)
    assert s["cases"] == 5 and s["p99_ms"] >= s["p50_ms"] > 0
