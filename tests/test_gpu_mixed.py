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
