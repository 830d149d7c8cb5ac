"""RANS{KOmega} on the GPU against the oracle (1e-10 relative L2, expected
0): the reference's transient k-omega backward-facing step (its own grid,
committed raw parse) host-polled and in graph mode, over 500 steps to its
known answer (outlet Ux = 0.5 inlet Ux within 0.1 Umag); a steady SIMPLE
k-omega channel with omega wall functions; k-omega cases refused by the
batch."""
import numpy as np
import pytest

from test_komega import KW_FIELDS, komega_bfs_case, set_komega_fields
from test_nonorth_oracle import skewed_channel
from test_unv import bfs_mesh

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


def _pair(x, orc, ctx, mesh, model, cfg, graph):
    dm = x.DeviceMesh(ctx, mesh)
    g = x.Case(dm, cfg)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    for c in (g, o):
        set_komega_fields(x, c, model)
    if graph:
        g.set_graph_mode(True)
    return g, o, dm


def _check(x, g, o, fields=KW_FIELDS + ("FIELD_NUTF", "FIELD_NUEFF", "FIELD_GRADU")):
    for f in fields:
        assert rel(g.get_field(getattr(x._abi, f)), o.get_field(getattr(x._abi, f))) <= TOL, f


@pytest.mark.parametrize("graph", [False, True])
def test_komega_bfs_parity(x, orc, ctx, graph):
    mesh = bfs_mesh(x, 5)
    model, config = komega_bfs_case(x, mesh, steps=10)
    cfg, keep = x.build_config(model, config)
    g, o, dm = _pair(x, orc, ctx, mesh, model, cfg, graph)
    rg, _ = g.piso_step(10)
    ro, _ = o.piso_step(10)
    assert rel(rg, ro) <= TOL, (rg, ro)
    _check(x, g, o)


def test_komega_bfs_known_answer_gpu(x, orc, ctx):
    mesh = bfs_mesh(x, 5)
    model, config = komega_bfs_case(x, mesh)
    cfg, keep = x.build_config(model, config)
    g, o, dm = _pair(x, orc, ctx, mesh, model, cfg, True)
    rg, _ = g.piso_step(500)
    ro, _ = o.piso_step(500)
    assert rel(rg, ro) <= TOL
    _check(x, g, o, KW_FIELDS)
    U = g.get_field(x._abi.FIELD_U)
    inlet = x.api.boundary_average("inlet", U, config.boundaries["U"], mesh=mesh)
    outlet = x.api.boundary_average("outlet", U, config.boundaries["U"], mesh=mesh)
    assert np.linalg.norm(outlet - 0.5 * inlet) <= 0.1 * 1.5, (inlet, outlet)


def komega_channel_case(x, mesh, iterations, precond="Jacobi", wallfn=False, sst=False):
    """Steady SIMPLE with RANS{KOmega} (or SST) on a 3D channel: k and omega
    Dirichlet at the inlet, Extrapolated at the outlet, omega wall functions
    on the walls, and k = nut = 0 there or (wallfn, nu 1e-5 so the wall
    cells sit in the log layer) k and nut wall functions."""
    A = x.api
    turb = A.RANS(A.KOmegaSST, walls=["walls"]) if sst else A.RANS(A.KOmega)
    model = A.Physics(time=A.Steady(), fluid=A.Fluid(A.Incompressible, nu=1e-5 if wallfn else 1e-3), turbulence=turb,
                      energy=A.Energy(A.Isothermal), domain=mesh)
    kw = A.KWallFunction("walls") if wallfn else A.Dirichlet("walls", 0.0)
    nw = A.NutWallFunction("walls") if wallfn else A.Dirichlet("walls", 0.0)
    BCs = A.assign(region=mesh,
                   U=[A.Dirichlet("inlet", [1.0, 0.0, 0.0]), A.Zerogradient("outlet"), A.Wall("walls", [0.0, 0.0, 0.0])],
                   p=[A.Zerogradient("inlet"), A.Dirichlet("outlet", 0.0), A.Wall("walls")],
                   k=[A.Dirichlet("inlet", 0.01), A.Extrapolated("outlet"), kw],
                   omega=[A.Dirichlet("inlet", 10.0), A.Extrapolated("outlet"), A.OmegaWallFunction("walls")],
                   nut=[A.Dirichlet("inlet", 1e-3), A.Extrapolated("outlet"), nw])
    pre = getattr(A, precond)

    def ss(s, relax):
        return A.SolverSetup(solver=s(), preconditioner=pre(), convergence=1e-7, relax=relax, rtol=1e-2)

    config = A.Configuration(solvers={"U": ss(A.Bicgstab, 0.7), "p": ss(A.Cg, 0.3), "k": ss(A.Bicgstab, 0.7),
                                      "omega": ss(A.Bicgstab, 0.7),
                                      "y": A.SolverSetup(solver=A.Cg(), preconditioner=A.Jacobi(), convergence=1e-8,
                                                         relax=0.9, rtol=1e-3)},
                             schemes={"U": A.Schemes(divergence=A.Upwind), "p": A.Schemes(),
                                      "k": A.Schemes(divergence=A.Upwind), "omega": A.Schemes(divergence=A.Upwind),
                                      "y": A.Schemes()},
                             runtime=A.Runtime(iterations=iterations, write_interval=-1, time_step=1.0),
                             hardware=A.Hardware(backend=A.B200Backend()), boundaries=BCs)
    A.initialise_(model.momentum.U, [1.0, 0.0, 0.0])
    A.initialise_(model.momentum.p, 0.0)
    A.initialise_(model.turbulence.k, 0.01)
    A.initialise_(model.turbulence.omega, 10.0)
    A.initialise_(model.turbulence.nut, 1e-3)
    return model, config


@pytest.mark.parametrize("precond", ["Jacobi", "DILU"])
def test_komega_simple_channel_parity(x, orc, ctx, precond):
    mesh = skewed_channel(x, n=(12, 7, 6), seed=11)
    model, config = komega_channel_case(x, mesh, 6, precond)
    cfg, keep = x.build_config(model, config)
    g, o, dm = _pair(x, orc, ctx, mesh, model, cfg, False)
    rg, _ = g.simple_iterate(6)
    ro, _ = o.simple_iterate(6)
    assert rel(rg, ro) <= TOL, (rg, ro)
    _check(x, g, o)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_komega_batch_matches_single(x, ctx, prec):
    """k-omega cases in a batch: their U and p solves batched with the other
    members', their k and omega solves each on its own stream; every case
    equals the same case advanced alone, bit for bit."""
    specs = [((12, 7, 6), 11, "Jacobi"), ((10, 6, 6), 3, "Jacobi")]

    def mk(n, seed):
        mesh = skewed_channel(x, n=n, seed=seed)
        model, config = komega_channel_case(x, mesh, 4)
        config.hardware.backend.precision = prec
        cfg, keep = x.build_config(model, config)
        dm = x.DeviceMesh(ctx, mesh)
        c = x.Case(dm, cfg)
        c.set_inner_cg(1)
        set_komega_fields(x, c, model)
        return c, (dm, keep, cfg)

    alone = []
    for n, seed, _ in specs:
        c, keep = mk(n, seed)
        res, _ = c.simple_iterate(4)
        alone.append((res, [c.get_field(getattr(x._abi, f)) for f in KW_FIELDS]))
    batch = x.api.Batch(ctx, 4, 1 << 32)
    members = []
    for n, seed, _ in specs:
        c, keep = mk(n, seed)
        assert batch.add(c)
        members.append((c, keep))
    hist = np.stack([batch.simple_iterate()[0] for _ in range(4)], axis=1)
    for k, (c, keep) in enumerate(members):
        assert np.array_equal(hist[k], alone[k][0]), k
        for f, ref in zip(KW_FIELDS, alone[k][1]):
            assert np.array_equal(c.get_field(getattr(x._abi, f)), ref), (k, f)
    batch.close()


def test_komega_restart_bit_identical(x, ctx):
    """checkpoint() / restore() carry k and omega: 4 + 4 steps from a
    restored case equal 8 steps in one go."""
    mesh = bfs_mesh(x, 5)

    def new_case():
        model, config = komega_bfs_case(x, mesh, steps=8)
        cfg, keep = x.build_config(model, config)
        dm = x.DeviceMesh(ctx, mesh)
        c = x.Case(dm, cfg)
        set_komega_fields(x, c, model)
        return c, (dm, keep)

    a, ka = new_case()
    ra = a.piso_step(8)[0]
    b, kb = new_case()
    rb = b.piso_step(4)[0]
    state = b.checkpoint()
    assert "FIELD_K" in state and "FIELD_OMEGA" in state
    c, kc = new_case()
    c.restore(state)
    rc = c.piso_step(4)[0]
    assert np.array_equal(np.concatenate([rb, rc]), ra)
    for f in KW_FIELDS:
        assert np.array_equal(c.get_field(getattr(x._abi, f)), a.get_field(getattr(x._abi, f))), f


@pytest.mark.parametrize("precond", ["Jacobi", "DILU"])
def test_sst_channel_parity(x, orc, ctx, precond):
    from test_komega import sst_channel_case
    mesh = skewed_channel(x, n=(12, 8, 7), seed=13)
    model, config = sst_channel_case(x, mesh, 6, precond)
    cfg, keep = x.build_config(model, config)
    g, o, dm = _pair(x, orc, ctx, mesh, model, cfg, False)
    assert rel(g.get_field(x._abi.FIELD_WALLDIST), o.get_field(x._abi.FIELD_WALLDIST)) <= TOL
    rg, _ = g.simple_iterate(6)
    ro, _ = o.simple_iterate(6)
    assert rel(rg, ro) <= TOL, (rg, ro)
    _check(x, g, o)


@pytest.mark.parametrize("graph", [False, True])
def test_sst_bfs_transient_parity(x, orc, ctx, graph):
    """PISO with k-omega SST on the 2D backward-facing step (walls: wall, top)."""
    from test_komega import sst_channel_case
    mesh = bfs_mesh(x, 10)
    model, config = sst_channel_case(x, mesh, 5, transient=True, walls=("wall", "top"))
    config.schemes["p"].gradient = x.api.Midpoint
    config.schemes["k"].gradient = x.api.Midpoint
    cfg, keep = x.build_config(model, config)
    g, o, dm = _pair(x, orc, ctx, mesh, model, cfg, graph)
    rg, _ = g.piso_step(5)
    ro, _ = o.piso_step(5)
    assert rel(rg, ro) <= TOL, (rg, ro)
    _check(x, g, o, KW_FIELDS + ("FIELD_WALLDIST", "FIELD_NUTF"))


@pytest.mark.parametrize("sst", [False, True])
def test_wall_functions_parity(x, orc, ctx, sst):
    """KWallFunction and NutWallFunction (log-law wall cells) with k-omega
    and k-omega SST."""
    mesh = skewed_channel(x, n=(12, 7, 6), seed=17)
    model, config = komega_channel_case(x, mesh, 6, wallfn=True, sst=sst)
    cfg, keep = x.build_config(model, config)
    g, o, dm = _pair(x, orc, ctx, mesh, model, cfg, False)
    rg, _ = g.simple_iterate(6)
    ro, _ = o.simple_iterate(6)
    assert rel(rg, ro) <= TOL, (rg, ro)
    _check(x, g, o)
    walls = list(mesh.patch_range("walls"))
    assert np.all(g.get_field(x._abi.FIELD_NUTF)[walls] > 0)  # the log-law branch ran


@pytest.mark.parametrize("sst", [False, True])
def test_komega_periodic_channel_parity(x, orc, ctx, sst):
    """k-omega (and SST) on a channel periodic in the flow direction (inlet
    and outlet paired by construct_periodic, every field periodic there),
    with a disturbed initial velocity and a pressure reference: the scalar
    equations' periodic pairs in the shared p storage; GPU equal to the
    oracle over 3 SIMPLE iterations."""
    A = x.api
    mesh = x.build_mesh3(x.channel_polymesh(12, 6, 6, seed=7))
    per = list(A.construct_periodic(mesh, None, "inlet", "outlet"))
    turb = A.RANS(A.KOmegaSST, walls=["walls"]) if sst else A.RANS(A.KOmega)
    model = A.Physics(time=A.Steady(), fluid=A.Fluid(A.Incompressible, nu=1e-3), turbulence=turb,
                      energy=A.Energy(A.Isothermal), domain=mesh)
    BCs = A.assign(region=mesh, U=per + [A.Wall("walls", [0.0, 0.0, 0.0])], p=per + [A.Wall("walls")],
                   k=per + [A.Dirichlet("walls", 0.0)], omega=per + [A.OmegaWallFunction("walls")],
                   nut=per + [A.Dirichlet("walls", 0.0)])

    def ss(s, relax):
        return A.SolverSetup(solver=s(), preconditioner=A.Jacobi(), convergence=1e-7, relax=relax, rtol=1e-2)

    config = A.Configuration(solvers={"U": ss(A.Bicgstab, 0.7), "p": ss(A.Cg, 0.3), "k": ss(A.Bicgstab, 0.7),
                                      "omega": ss(A.Bicgstab, 0.7),
                                      "y": A.SolverSetup(solver=A.Cg(), preconditioner=A.Jacobi(), convergence=1e-8,
                                                         relax=0.9, rtol=1e-3)},
                             schemes={"U": A.Schemes(divergence=A.Upwind), "p": A.Schemes(),
                                      "k": A.Schemes(divergence=A.Upwind), "omega": A.Schemes(divergence=A.Upwind),
                                      "y": A.Schemes()},
                             runtime=A.Runtime(iterations=3, write_interval=-1, time_step=1.0),
                             hardware=A.Hardware(backend=A.B200Backend()), boundaries=BCs)
    rng = np.random.default_rng(7)
    model.momentum.U[:] = np.array([[1.0], [0.0], [0.0]]) + 0.05 * rng.standard_normal((3, mesh.n_cells))
    A.initialise_(model.momentum.p, 0.0)
    A.initialise_(model.turbulence.k, 0.01)
    A.initialise_(model.turbulence.omega, 10.0)
    A.initialise_(model.turbulence.nut, 1e-3)
    cfg, keep = x.build_config(model, config, pref=0.0)
    g, o, dm = _pair(x, orc, ctx, mesh, model, cfg, False)
    rg, _ = g.simple_iterate(3)
    ro, _ = o.simple_iterate(3)
    assert rel(rg, ro) <= TOL, (rg, ro)
    _check(x, g, o)


def test_komega_dilu_k_jacobi_p_parity(x, orc, ctx):
    """k and omega DILU-preconditioned while p is Jacobi: the p system's
    storage, which k and omega share, carries the DILU levels their solves
    need.  GPU equal to the oracle."""
    mesh = skewed_channel(x, n=(12, 7, 6), seed=11)
    model, config = komega_channel_case(x, mesh, 6, "DILU")
    A = x.api
    config.solvers["p"] = A.SolverSetup(solver=A.Cg(), preconditioner=A.Jacobi(), convergence=1e-7, relax=0.3,
                                        rtol=1e-2)
    cfg, keep = x.build_config(model, config)
    assert cfg.p_solver.precond == x._abi.PRECOND_JACOBI and cfg.k_solver.precond == x._abi.PRECOND_DILU
    g, o, dm = _pair(x, orc, ctx, mesh, model, cfg, False)
    rg, _ = g.simple_iterate(6)
    ro, _ = o.simple_iterate(6)
    assert rel(rg, ro) <= TOL, (rg, ro)
    _check(x, g, o)
