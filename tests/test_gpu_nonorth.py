"""Non-orthogonal correctors, Midpoint gradients and the CellBased, FaceBased and MFaceBased
gradient limiters on the GPU against the oracle (skewed channel, FP64, host-polled and
graph mode; tolerance the 1e-10 relative L2 of the parity tests, expected 0),
and a batch of skewed cases with correctors (and limiters) giving the results
the cases give alone (bit for bit)."""
import numpy as np
import pytest

from test_nonorth_oracle import skewed_channel

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("ncorr", [1, 2])
def test_correctors_parity(x, orc, ctx, ncorr, graph):
    mesh = skewed_channel(x, n=(12, 7, 6), seed=4)
    model, config = x.cases.channel_case(mesh, iterations=4)
    cfg, keep = x.build_config(model, config, ncorrectors=ncorr)
    dm = x.DeviceMesh(ctx, mesh)
    g = x.Case(dm, cfg)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    for c in (g, o):
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
    if graph:
        g.set_graph_mode(True)
    rg, _ = g.simple_iterate(4)
    ro, _ = o.simple_iterate(4)
    assert rel(rg, ro) <= TOL, (rg, ro)
    for f in (x._abi.FIELD_U, x._abi.FIELD_P, x._abi.FIELD_MDOTF):
        assert rel(g.get_field(f), o.get_field(f)) <= TOL


@pytest.mark.parametrize("limit", [False, True])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_correctors_batch_matches_single(x, ctx, prec, limit):
    specs = [((10, 6, 5), 3), ((14, 8, 7), 5), ((9, 9, 4), 6)]
    iters = 3

    def mk(n, seed):
        mesh = skewed_channel(x, n=n, seed=seed)
        model, config = x.cases.channel_case(mesh, iterations=iters, precision=prec)
        if limit:
            config.schemes["p"].limiter = x.api.CellBased(1.0)
            config.schemes["U"].limiter = x.api.CellBased(0.7)
        cfg, keep = x.build_config(model, config, ncorrectors=2)
        dm = x.DeviceMesh(ctx, mesh)
        c = x.Case(dm, cfg)
        c.set_inner_cg(1)  # the batch's FP32 inner CG form (a case takes it when admitted)
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
        return c, (dm, keep)

    alone = []
    for n, seed in specs:
        c, keep = mk(n, seed)
        res, _ = c.simple_iterate(iters)
        alone.append((res, c.get_field(x._abi.FIELD_P)))
    batch = x.api.Batch(ctx, 4, 1 << 34)
    members = [mk(n, seed) for n, seed in specs]
    for c, _ in members:
        assert batch.add(c)
    hist = np.stack([batch.simple_iterate()[0] for _ in range(iters)], axis=1)
    for k, (c, _) in enumerate(members):
        assert np.array_equal(hist[k], alone[k][0]), (k, hist[k], alone[k][0])
        assert np.array_equal(c.get_field(x._abi.FIELD_P), alone[k][1])
    batch.close()


@pytest.mark.parametrize("which,ncorr", [("p", 0), ("pU", 0), ("pU", 1)])
def test_midpoint_gradient_parity(x, orc, ctx, which, ncorr):
    """Midpoint gradients (grad p; grad p and grad U) on the skewed channel,
    with and without a non-orthogonal corrector: GPU against the oracle."""
    mesh = skewed_channel(x, n=(11, 7, 6), seed=8)
    model, config = x.cases.channel_case(mesh, iterations=4)
    config.schemes["p"].gradient = x.api.Midpoint
    if "U" in which:
        config.schemes["U"].gradient = x.api.Midpoint
    cfg, keep = x.build_config(model, config, ncorrectors=ncorr)
    dm = x.DeviceMesh(ctx, mesh)
    g = x.Case(dm, cfg)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    for c in (g, o):
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
    rg, _ = g.simple_iterate(4)
    ro, _ = o.simple_iterate(4)
    assert rel(rg, ro) <= TOL, (rg, ro)
    for f in (x._abi.FIELD_U, x._abi.FIELD_P, x._abi.FIELD_GRADP, x._abi.FIELD_GRADU):
        assert rel(g.get_field(f), o.get_field(f)) <= TOL, f


def test_midpoint_les_piso_parity(x, orc, ctx):
    """PISO + Smagorinsky with Midpoint grad U (nut from the last pass) and
    grad p on the periodic box: GPU against the oracle."""
    mesh = x.build_mesh3(x.periodic_box_polymesh(8, seed=3))
    U0 = x.cases.fourier_field(mesh, seed=3)
    model, config = x.cases.periodic_les_case(mesh, steps=3, U0=U0)
    config.schemes["p"].gradient = x.api.Midpoint
    config.schemes["U"].gradient = x.api.Midpoint
    cfg, keep = x.build_config(model, config, pref=0.0)
    dm = x.DeviceMesh(ctx, mesh)
    g = x.Case(dm, cfg)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    for c in (g, o):
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
    rg, _ = g.piso_step(3)
    ro, _ = o.piso_step(3)
    assert rel(rg, ro) <= TOL, (rg, ro)
    for f in (x._abi.FIELD_U, x._abi.FIELD_P, x._abi.FIELD_NUT):
        assert rel(g.get_field(f), o.get_field(f)) <= TOL, f


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("grad,p_level,U_level,ncorr", [("gauss", 1.0, None, 0), ("gauss", 1.0, 1.0, 1),
                                                        ("midpoint", 0.5, 0.8, 1)])
def test_limiter_parity(x, orc, ctx, grad, p_level, U_level, ncorr, graph):
    """Schemes(limiter=CellBased(level)) for p (and U) on the skewed channel,
    Gauss or Midpoint gradients, with and without a corrector."""
    mesh = skewed_channel(x, n=(12, 7, 6), seed=9)
    model, config = x.cases.channel_case(mesh, iterations=4)
    config.schemes["p"].limiter = x.api.CellBased(p_level)
    if U_level is not None:
        config.schemes["U"].limiter = x.api.CellBased(U_level)
    if grad == "midpoint":
        config.schemes["p"].gradient = x.api.Midpoint
        config.schemes["U"].gradient = x.api.Midpoint
    cfg, keep = x.build_config(model, config, ncorrectors=ncorr)
    dm = x.DeviceMesh(ctx, mesh)
    g = x.Case(dm, cfg)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    for c in (g, o):
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
    if graph:
        g.set_graph_mode(True)
    rg, _ = g.simple_iterate(4)
    ro, _ = o.simple_iterate(4)
    assert rel(rg, ro) <= TOL, (rg, ro)
    for f in (x._abi.FIELD_U, x._abi.FIELD_P, x._abi.FIELD_GRADP, x._abi.FIELD_GRADU):
        assert rel(g.get_field(f), o.get_field(f)) <= TOL, f



@pytest.mark.parametrize("kind", ["FaceBased", "MFaceBased"])
@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("grad", ["gauss", "midpoint"])
def test_face_limiter_parity(x, orc, ctx, grad, graph, kind):
    """Schemes(limiter=FaceBased / MFaceBased) for p (scalar form) and U
    (tensor form) on the skewed channel with a corrector: GPU equal to the
    oracle."""
    mesh = skewed_channel(x, n=(12, 7, 6), seed=10)
    model, config = x.cases.channel_case(mesh, iterations=4)
    config.schemes["p"].limiter = getattr(x.api, kind)(mesh)
    config.schemes["U"].limiter = getattr(x.api, kind)(mesh)
    if grad == "midpoint":
        config.schemes["p"].gradient = x.api.Midpoint
        config.schemes["U"].gradient = x.api.Midpoint
    cfg, keep = x.build_config(model, config, ncorrectors=1)
    dm = x.DeviceMesh(ctx, mesh)
    g = x.Case(dm, cfg)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    for c in (g, o):
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
    if graph:
        g.set_graph_mode(True)
    rg, _ = g.simple_iterate(4)
    ro, _ = o.simple_iterate(4)
    assert rel(rg, ro) <= TOL, (rg, ro)
    for f in (x._abi.FIELD_U, x._abi.FIELD_P, x._abi.FIELD_GRADP, x._abi.FIELD_GRADU):
        assert rel(g.get_field(f), o.get_field(f)) <= TOL, f

def test_limiter_les_piso_parity(x, orc, ctx):
    """PISO + Smagorinsky with the grad U limiter (nut from the limited
    gradient, LES_Smagorinsky.jl:119-127) and the grad p limiter."""
    mesh = x.build_mesh3(x.periodic_box_polymesh(8, seed=4))
    U0 = x.cases.fourier_field(mesh, seed=4)
    model, config = x.cases.periodic_les_case(mesh, steps=3, U0=U0)
    config.schemes["p"].limiter = x.api.CellBased(1.0)
    config.schemes["U"].limiter = x.api.CellBased(1.0)
    cfg, keep = x.build_config(model, config, pref=0.0)
    dm = x.DeviceMesh(ctx, mesh)
    g = x.Case(dm, cfg)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    for c in (g, o):
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
    rg, _ = g.piso_step(3)
    ro, _ = o.piso_step(3)
    assert rel(rg, ro) <= TOL, (rg, ro)
    for f in (x._abi.FIELD_U, x._abi.FIELD_P, x._abi.FIELD_NUT, x._abi.FIELD_GRADU):
        assert rel(g.get_field(f), o.get_field(f)) <= TOL, f


@pytest.mark.parametrize("kind", ["FaceBased", "MFaceBased"])
def test_face_limiters_batch_matches_single(x, ctx, kind):
    """The face-based limiters (p and U) in a batch with a corrector: each
    case equals the same case advanced alone, bit for bit."""
    specs = [((10, 6, 5), 3), ((12, 7, 6), 5)]
    iters = 3

    def mk(n, seed):
        mesh = skewed_channel(x, n=n, seed=seed)
        model, config = x.cases.channel_case(mesh, iterations=iters)
        config.schemes["p"].limiter = getattr(x.api, kind)(mesh)
        config.schemes["U"].limiter = getattr(x.api, kind)(mesh)
        cfg, keep = x.build_config(model, config, ncorrectors=1)
        dm = x.DeviceMesh(ctx, mesh)
        c = x.Case(dm, cfg)
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
        return c, (dm, keep)

    alone = []
    for n, seed in specs:
        c, keep = mk(n, seed)
        res, _ = c.simple_iterate(iters)
        alone.append((res, c.get_field(x._abi.FIELD_P), c.get_field(x._abi.FIELD_GRADU)))
    batch = x.api.Batch(ctx, 4, 1 << 32)
    members = [mk(n, seed) for n, seed in specs]
    for c, _ in members:
        assert batch.add(c)
    hist = np.stack([batch.simple_iterate()[0] for _ in range(iters)], axis=1)
    for k, (c, _) in enumerate(members):
        assert np.array_equal(hist[k], alone[k][0]), k
        assert np.array_equal(c.get_field(x._abi.FIELD_P), alone[k][1])
        assert np.array_equal(c.get_field(x._abi.FIELD_GRADU), alone[k][2])
    batch.close()
