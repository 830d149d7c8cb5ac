"""GPU parity tests: every step of the SIMPLE path through the C ABI against
the CPU oracle on the same seeded inputs.

Tolerance: the device reproduces the oracle's operation order (no FMA
contraction, fixed reduction trees), so the expected difference is zero; the
asserted bound is the 1e-10 relative L2 of the FP64 parity target.
"""
import numpy as np
import pytest

from test_oracle_golden import laplace_check, laplace_setup

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def make_pair(x, orc, ctx, mesh, model, config, pref=None):
    cfg, keep = x.build_config(model, config, pref=pref)
    dm = x.DeviceMesh(ctx, mesh)
    g = x.Case(dm, cfg)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    for c in (g, o):
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
    return g, o, (cfg, keep, dm)


FIELDS = ["FIELD_U", "FIELD_P", "FIELD_MDOTF", "FIELD_NUEFF", "FIELD_GRADP", "FIELD_GRADU", "FIELD_RD", "FIELD_HV",
          "FIELD_DIVHV", "FIELD_UF", "FIELD_PF", "FIELD_RDF"]


def compare_fields(x, g, o, names=FIELDS, tol=TOL):
    bad = {}
    for n in names:
        fid = getattr(x._abi, n)
        e = rel(g.get_field(fid), o.get_field(fid))
        if not e <= tol:
            bad[n] = e
    assert not bad, bad


def channel(x, n=(10, 6, 5), seed=4, iters=5):
    mesh = x.build_mesh3(x.channel_polymesh(*n, seed=seed))
    model, config = x.cases.channel_case(mesh, iterations=iters)
    return mesh, model, config


def test_pattern_bitexact(x, orc, ctx):
    mesh, model, config = channel(x)
    g, o, keep = make_pair(x, orc, ctx, mesh, model, config)
    for eqn in (0, 1):
        rg, cg = g.pattern(eqn)
        ro, co = o.pattern(eqn)
        assert np.array_equal(rg, ro) and np.array_equal(cg, co)


def test_laplace_golden_gpu(x, orc, ctx):
    m, cfg, keep = laplace_setup(x)
    dm = x.DeviceMesh(ctx, m)
    g = x.Case(dm, cfg)
    g.discretise(1)
    g.apply_boundary_conditions(1)
    rp, cv = g.pattern(1)
    nz, b = g.system(1)
    laplace_check(m, nz, rp, cv, b)


def test_stepwise_simple_parity(x, orc, ctx):
    mesh, model, config = channel(x)
    rng = np.random.default_rng(0)
    model.momentum.U[:] = rng.standard_normal(model.momentum.U.shape) * 0.1
    model.momentum.p[:] = rng.standard_normal(model.momentum.p.shape) * 0.01
    g, o, keep = make_pair(x, orc, ctx, mesh, model, config)
    for c in (g, o):
        c.initial_calculations()
    compare_fields(x, g, o, ["FIELD_UF", "FIELD_MDOTF", "FIELD_PF", "FIELD_GRADP", "FIELD_NUEFF"], tol=0.0)
    # momentum assembly (A0, bx)
    for c in (g, o):
        c.discretise(0)
    ng, bg = g.system(0, -1)
    no, bo = o.system(0, -1)
    assert rel(ng, no) == 0.0 and rel(bg, bo) == 0.0
    # BCs + relaxation per component, solves
    for d in range(3):
        for c in (g, o):
            c.apply_boundary_conditions(0, d)
        ng, bg = g.system(0, d)
        no, bo = o.system(0, d)
        assert rel(ng, no) == 0.0 and rel(bg, bo) == 0.0, d
        for c in (g, o):
            c.implicit_relaxation_diagdom(d)
            if d == 0:
                c.update_preconditioner(0)
        ng, bg = g.system(0, d)
        no, bo = o.system(0, d)
        assert rel(ng, no) == 0.0 and rel(bg, bo) == 0.0, d
        rg, ig = g.solve_system(0, d)
        ro, io = o.solve_system(0, d)
        assert ig == io and rg == ro, (d, ig, io, rg, ro)
    compare_fields(x, g, o, ["FIELD_U"], tol=0.0)
    for c in (g, o):
        c.pressure_predictor()
    compare_fields(x, g, o, ["FIELD_RD", "FIELD_RDF", "FIELD_HV"], tol=0.0)
    for c in (g, o):
        c.flux_divergence()
    compare_fields(x, g, o, ["FIELD_UF", "FIELD_MDOTF", "FIELD_DIVHV"], tol=0.0)
    rg = g.solve_equation(1)
    ro = o.solve_equation(1)
    assert rg == ro
    ng, bg = g.system(1)
    no, bo = o.system(1)
    assert rel(ng, no) == 0.0 and rel(bg, bo) == 0.0
    for c in (g, o):
        c.explicit_relaxation_p(0.3)
        c.grad_p()
        c.correct()
        c.turbulence()
    compare_fields(x, g, o, FIELDS, tol=0.0)


@pytest.mark.parametrize("kind", ["channel", "cavity"])
def test_simple_iterations_parity(x, orc, ctx, kind):
    if kind == "channel":
        mesh, model, config = channel(x, n=(16, 8, 8), seed=9, iters=8)
        pref = None
    else:
        mesh = x.build_mesh3(x.cavity_polymesh(24))
        model, config = x.cases.cavity_case(mesh, iterations=8)
        pref = 0.0
    g, o, keep = make_pair(x, orc, ctx, mesh, model, config, pref=pref)
    rg, cg = g.simple_iterate(8)
    ro, co = o.simple_iterate(8)
    assert rg.shape == ro.shape
    assert rel(rg, ro) <= TOL, (rg, ro)
    compare_fields(x, g, o)


def test_determinism_two_runs(x, ctx):
    mesh, model, config = channel(x, n=(20, 10, 10), seed=2, iters=3)
    out = []
    for _ in range(2):
        cfg, keep = x.build_config(model, config)
        dm = x.DeviceMesh(ctx, mesh)
        g = x.Case(dm, cfg)
        res, _ = g.simple_iterate(3)
        out.append((res, g.get_field(x._abi.FIELD_U), g.get_field(x._abi.FIELD_P)))
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
    # reading into a caller's buffer (get_field(out=)) gives the same values
    U = np.empty((3, mesh.n_cells))
    p = np.empty(mesh.n_cells)
    assert g.get_field(x._abi.FIELD_U, out=U) is U and g.get_field(x._abi.FIELD_P, out=p) is p
    assert np.array_equal(U, out[1][1]) and np.array_equal(p, out[1][2])
    with pytest.raises(ValueError):
        g.get_field(x._abi.FIELD_P, out=np.empty(mesh.n_cells, dtype=np.float32))


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_dilu_modes_parity(x, orc, ctx, mode):
    """Momentum DILU as one-block sweeps, as per-level kernels over the
    level-ordered triangles, and as one cooperative launch over every level:
    each equals the oracle bit for bit."""
    mesh = x.build_mesh3(x.channel_polymesh(34, 44, 46, seed=12))   # 68,816 cells
    model, config = x.cases.channel_case(mesh, iterations=2)
    g, o, keep = make_pair(x, orc, ctx, mesh, model, config)
    g.set_dilu_mode(mode)
    rg, cg = g.simple_iterate(2)
    ro, co = o.simple_iterate(2)
    assert rel(rg, ro) <= TOL, (rg, ro)
    compare_fields(x, g, o, ["FIELD_U", "FIELD_P"], tol=0.0)


def test_dilu_grid_mixed_identical(x, ctx):
    """Mixed precision: the FP32 momentum DILU as one-block sweeps (next
    level's rows loaded before each barrier), as per-level kernels and as one
    cooperative launch over every level give the same run bit for bit."""
    mesh = x.build_mesh3(x.channel_polymesh(40, 30, 30, seed=8))
    out = []
    for mode in (1, 2, 3):
        model, config = x.cases.channel_case(mesh, iterations=3, precision="mixed")
        cfg, keep = x.build_config(model, config)
        dm = x.DeviceMesh(ctx, mesh)
        g = x.Case(dm, cfg)
        g.set_field(x._abi.FIELD_U, model.momentum.U)
        g.set_field(x._abi.FIELD_P, model.momentum.p)
        g.set_dilu_mode(mode)
        res, _ = g.simple_iterate(3)
        out.append((res, g.get_field(x._abi.FIELD_U), g.get_field(x._abi.FIELD_P)))
        g.close()
        dm.close()
    for o in out[1:]:
        for a, b in zip(out[0], o):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("graph", [False, True])
def test_neumann_p_parity(x, orc, ctx, graph):
    """p with a Neumann inlet (neumann.jl, scalar: a fixed normal gradient in
    the face value, the Laplacian's boundary source and the interpolation)
    through SIMPLE: GPU equal to the oracle, host-polled and in graph mode."""
    mesh = x.build_mesh3(x.channel_polymesh(12, 7, 6, seed=6))
    model, config = x.cases.channel_case(mesh, iterations=4)
    config.boundaries["p"] = x.api.assign(region=mesh, p=[x.api.Neumann("inlet", 0.05), x.api.Dirichlet("outlet", 0.0),
                                                           x.api.Wall("walls")])["p"]
    g, o, keep = make_pair(x, orc, ctx, mesh, model, config)
    if graph:
        g.set_graph_mode(True)
    rg, _ = g.simple_iterate(4)
    ro, _ = o.simple_iterate(4)
    assert rel(rg, ro) <= TOL, (rg, ro)
    compare_fields(x, g, o)
