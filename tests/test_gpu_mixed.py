"""Mixed precision (FP32 Krylov inner solves inside FP64 defect correction)
against the plain FP64 GPU path, which is the oracle for reduced precision.

Stated tolerances:
  * one pressure solve with rtol = 1e-9: relative L2 of p <= 1e-6
    (both stop on the same monitored-norm target; the bound covers the
    conditioning of the 7-point system);
  * a steady case converged to a 1e-6 scaled residual in both modes:
    relative L2 of U and p <= 1e-5.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _case(x, ctx, mesh, model, config, pref=None):
    cfg, keep = x.build_config(model, config, pref=pref)
    dm = x.DeviceMesh(ctx, mesh)
    c = x.Case(dm, cfg)
    c.set_field(x._abi.FIELD_U, model.momentum.U)
    c.set_field(x._abi.FIELD_P, model.momentum.p)
    return c, (cfg, keep, dm)


def test_mixed_pressure_solve_tight(x, ctx):
    mesh = x.build_mesh3(x.channel_polymesh(16, 8, 8, seed=3))
    out = {}
    for prec in ("fp64", "mixed"):
        model, config = x.cases.channel_case(mesh, iterations=3, precision=prec)
        config.solvers["p"].rtol = 1e-9
        rng = np.random.default_rng(1)
        model.momentum.U[:] = rng.standard_normal(model.momentum.U.shape) * 0.1
        c, keep = _case(x, ctx, mesh, model, config)
        c.initial_calculations()
        c.solve_equation(0)
        c.pressure_predictor()
        c.flux_divergence()
        res = c.solve_equation(1)
        out[prec] = (c.get_field(x._abi.FIELD_P), c.get_field(x._abi.FIELD_U), res)
    assert rel(out["mixed"][0], out["fp64"][0]) <= 1e-6
    # the momentum predictor ran with rtol 0.1 in both modes: same target,
    # different Krylov trajectories
    assert rel(out["mixed"][1], out["fp64"][1]) <= 5e-2


def test_mixed_converged_cavity_matches_fp64(x, ctx):
    mesh = x.build_mesh3(x.cavity_polymesh(16))
    out = {}
    for prec in ("fp64", "mixed"):
        model, config = x.cases.cavity_case(mesh, iterations=3000, precision=prec)
        for s in ("U", "p"):
            config.solvers[s].convergence = 1e-6
        c, keep = _case(x, ctx, mesh, model, config, pref=0.0)
        res, conv = c.simple_iterate(3000)
        assert conv, (prec, res[-1])
        out[prec] = (c.get_field(x._abi.FIELD_U), c.get_field(x._abi.FIELD_P), len(res))
    assert rel(out["mixed"][0], out["fp64"][0]) <= 1e-5, rel(out["mixed"][0], out["fp64"][0])
    assert rel(out["mixed"][1], out["fp64"][1]) <= 1e-5, rel(out["mixed"][1], out["fp64"][1])


def _tight_pressure(x, ctx, mesh, prec, inner_cg=None):
    """One pressure solve to rtol 1e-9 after a momentum predictor from a
    seeded velocity; returns p."""
    model, config = x.cases.channel_case(mesh, iterations=3, precision=prec)
    config.solvers["p"].rtol = 1e-9
    rng = np.random.default_rng(1)
    model.momentum.U[:] = rng.standard_normal(model.momentum.U.shape) * 0.1
    c, keep = _case(x, ctx, mesh, model, config)
    if inner_cg is not None:
        c.set_inner_cg(inner_cg)
    c.initial_calculations()
    c.solve_equation(0)
    c.pressure_predictor()
    c.flux_divergence()
    c.solve_equation(1)
    p = c.get_field(x._abi.FIELD_P)
    c.close()
    keep[2].close()
    return p


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4, 5, 13])
def test_inner_cg_forms_tight(x, ctx, mode):
    """Every form of the FP32 inner CG (Jacobi-scaled system in each launch
    shape; the canonical kernels) meets the tight-solve bound against FP64."""
    mesh = x.build_mesh3(x.channel_polymesh(24, 12, 12, seed=3))
    p64 = _tight_pressure(x, ctx, mesh, "fp64")
    p = _tight_pressure(x, ctx, mesh, "mixed", inner_cg=mode)
    assert rel(p, p64) <= 1e-6, rel(p, p64)


@pytest.mark.parametrize("form", [0, 1, 2, 3])
def test_inner_cg_layouts_identical(x, ctx, form):
    """The scaled-system kernel with x and p in global memory (the layout
    of systems too large for shared memory), with per-slice slot widths (the
    layout of meshes whose rows differ widely in length), and with both,
    gives the default layout's result bit for bit: only where data lives
    differs.  Shapes of the same thread count (0 and 2, 1 and 3) agree bit
    for bit as well."""
    mesh = x.build_mesh3(x.channel_polymesh(40, 24, 20, seed=4))
    a = _tight_pressure(x, ctx, mesh, "mixed", inner_cg=2 + form)
    for extra in (4, 8, 12):
        b = _tight_pressure(x, ctx, mesh, "mixed", inner_cg=2 + form + extra)
        assert np.array_equal(a, b), extra
    same_nt = {0: 2, 1: 3, 2: 0, 3: 1}[form]
    b = _tight_pressure(x, ctx, mesh, "mixed", inner_cg=2 + same_nt)
    assert np.array_equal(a, b), same_nt


def test_inner_cg_graph_mode_identical(x, ctx):
    """The scaled-system inner CG captured in a step graph gives the
    host-polled run's results bit for bit (deterministic reductions)."""
    mesh = x.build_mesh3(x.channel_polymesh(20, 10, 10, seed=6))
    out = []
    for graph in (False, True):
        model, config = x.cases.channel_case(mesh, iterations=4, precision="mixed")
        c, keep = _case(x, ctx, mesh, model, config)
        c.set_graph_mode(graph)
        res, _ = c.simple_iterate(4)
        out.append((res, c.get_field(x._abi.FIELD_U), c.get_field(x._abi.FIELD_P)))
        c.close()
        keep[2].close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
