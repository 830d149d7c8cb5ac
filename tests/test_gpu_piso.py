"""GPU parity of the transient path: PISO + Smagorinsky LES, periodic boxes
(construct_periodic pairs on all three axes) and a walled channel, through
the C ABI against the CPU oracle on the same seeded inputs.

Tolerance: the device follows the oracle's operation order, so differences
are expected to be zero; the asserted bound is the 1e-10 relative L2 of the
FP64 parity target.
"""
import numpy as np
import pytest

from test_gpu_parity import FIELDS, compare_fields, make_pair, rel

pytestmark = pytest.mark.gpu

TOL = 1e-10
LES_FIELDS = FIELDS + ["FIELD_NUT", "FIELD_NUTF"]


def periodic(x, n=8, seed=5, steps=3):
    mesh = x.build_mesh3(x.periodic_box_polymesh(n, seed=seed))
    U0 = x.cases.fourier_field(mesh, seed=seed)
    model, config = x.cases.periodic_les_case(mesh, steps=steps, U0=U0)
    return mesh, model, config


def test_periodic_pattern_bitexact(x, orc, ctx):
    mesh, model, config = periodic(x)
    g, o, keep = make_pair(x, orc, ctx, mesh, model, config, pref=0.0)
    for eqn in (0, 1):
        rg, cg = g.pattern(eqn)
        ro, co = o.pattern(eqn)
        assert np.array_equal(rg, ro) and np.array_equal(cg, co)


def test_periodic_systems_after_bcs(x, orc, ctx):
    """Assembled U and p systems with the periodic matrix terms applied."""
    mesh, model, config = periodic(x)
    g, o, keep = make_pair(x, orc, ctx, mesh, model, config, pref=0.0)
    for c in (g, o):
        c.initial_calculations()
        c.turbulence()
        c.discretise(0)
    for d in range(3):
        for c in (g, o):
            c.apply_boundary_conditions(0, d)
        ng, bg = g.system(0, d)
        no, bo = o.system(0, d)
        assert rel(ng, no) == 0.0 and rel(bg, bo) == 0.0, d
    ng, bg = g.system(0, -1)
    no, bo = o.system(0, -1)
    assert rel(ng, no) == 0.0 and rel(bg, bo) == 0.0
    for c in (g, o):
        c.pressure_predictor()
        c.flux_divergence()
        c.discretise(1)
        c.apply_boundary_conditions(1)
        c.set_reference()
    ng, bg = g.system(1)
    no, bo = o.system(1)
    assert rel(ng, no) == 0.0 and rel(bg, bo) == 0.0


def test_piso_les_periodic_parity(x, orc, ctx):
    mesh, model, config = periodic(x, steps=3)
    g, o, keep = make_pair(x, orc, ctx, mesh, model, config, pref=0.0)
    rg, cog = g.piso_step(3)
    ro, coo = o.piso_step(3)
    assert rg.shape == ro.shape == (3, 4)
    assert rel(rg, ro) <= TOL, (rg, ro)
    assert rel(cog, coo) <= TOL, (cog, coo)
    compare_fields(x, g, o, LES_FIELDS)


def test_piso_les_channel_parity(x, orc, ctx):
    """Walled channel, transient LES (no periodic pair): Smagorinsky with a
    DirichletFunction inlet and zero-gradient outlet."""
    A = x.api
    mesh = x.build_mesh3(x.channel_polymesh(12, 6, 6, seed=7))
    model = A.Physics(time=A.Transient(), fluid=A.Fluid(A.Incompressible, nu=1e-4),
                      turbulence=A.LES(A.Smagorinsky, C=0.17), energy=A.Energy(A.Isothermal), domain=mesh)
    BCs = A.assign(
        region=mesh,
        U=[A.DirichletFunction("inlet", x.cases.parabolic_inlet), A.Zerogradient("outlet"),
           A.Wall("walls", [0.0, 0.0, 0.0])],
        p=[A.Zerogradient("inlet"), A.Dirichlet("outlet", 0.0), A.Wall("walls")],
        nut=[A.Zerogradient("inlet"), A.Zerogradient("outlet"), A.Dirichlet("walls", 0.0)],
    )
    schemes = {"U": A.Schemes(time=A.Euler, divergence=A.LUST), "p": A.Schemes(time=A.Euler)}
    solvers = x.cases._solvers(relax_U=1.0, relax_p=1.0, rtol_U=0.1, rtol_p=0.01)
    config = A.Configuration(solvers=solvers, schemes=schemes,
                             runtime=A.Runtime(iterations=4, write_interval=-1, time_step=0.01),
                             hardware=A.Hardware(backend=A.B200Backend()), boundaries=BCs)
    rng = np.random.default_rng(3)
    model.momentum.U[0] = 0.5 + 0.05 * rng.standard_normal(mesh.n_cells)
    g, o, keep = make_pair(x, orc, ctx, mesh, model, config)
    rg, cog = g.piso_step(4)
    ro, coo = o.piso_step(4)
    assert rel(rg, ro) <= TOL, (rg, ro)
    assert rel(cog, coo) <= TOL
    compare_fields(x, g, o, LES_FIELDS)


def test_piso_mixed_close_to_fp64(x, ctx):
    """Mixed precision on the transient periodic case: fields within 1e-5
    relative L2 of the FP64 GPU path after 5 steps (pressure rtol 1e-6)."""
    mesh = x.build_mesh3(x.periodic_box_polymesh(10, seed=2))
    U0 = x.cases.fourier_field(mesh, seed=2)
    out = {}
    for prec in ("fp64", "mixed"):
        model, config = x.cases.periodic_les_case(mesh, steps=5, U0=U0, precision=prec)
        config.solvers["p"].rtol = 1e-6
        config.solvers["U"].rtol = 1e-6
        cfg, keep = x.build_config(model, config, pref=0.0)
        dm = x.DeviceMesh(ctx, mesh)
        c = x.Case(dm, cfg)
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
        c.piso_step(5)
        out[prec] = (c.get_field(x._abi.FIELD_U), c.get_field(x._abi.FIELD_P))
    assert rel(out["mixed"][0], out["fp64"][0]) <= 1e-5
    assert rel(out["mixed"][1], out["fp64"][1]) <= 1e-5
