"""Non-orthogonal correctors (run!(...; ncorrectors), Solvers_1_SIMPLE.jl:
196-206, 267-333) on the CPU oracle: on a skewed channel (interior points
moved, faces up to ~27 degrees non-orthogonal) the corrector loop runs,
stays finite and changes the pressure solution."""
import numpy as np
import pytest


def skewed_channel(x, n=(10, 6, 5), seed=3, skew=0.2):
    pm = x.box_polymesh(*n, lengths=(2.0, 1.0, 1.0), seed=seed, skew=skew, skew_seed=seed,
                        patches=[("inlet", ["xmin"]), ("outlet", ["xmax"]), ("walls", ["ymin", "ymax", "zmin", "zmax"])])
    return x.build_mesh3(pm)


@pytest.mark.parametrize("ncorr", [1, 2])
def test_correctors_run_and_act(x, orc, ncorr):
    mesh = skewed_channel(x)
    out = {}
    for k in (0, ncorr):
        model, config = x.cases.channel_case(mesh, iterations=5)
        cfg, keep = x.build_config(model, config, ncorrectors=k)
        o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
        o.set_field(x._abi.FIELD_U, model.momentum.U)
        o.set_field(x._abi.FIELD_P, model.momentum.p)
        res, _ = o.simple_iterate(5)
        out[k] = (res, o.get_field(x._abi.FIELD_P))
    assert np.all(np.isfinite(out[ncorr][0]))
    assert not np.array_equal(out[0][1], out[ncorr][1])


def test_midpoint_gradient_acts(x, orc):
    """Schemes(gradient=Midpoint) (Calculate_0_gradient.jl:170-262) on the
    skewed channel: runs, stays finite, and differs from Gauss."""
    mesh = skewed_channel(x)
    out = {}
    for grad in ("gauss", "midpoint"):
        model, config = x.cases.channel_case(mesh, iterations=4)
        if grad == "midpoint":
            config.schemes["p"].gradient = x.api.Midpoint
            config.schemes["U"].gradient = x.api.Midpoint
        cfg, keep = x.build_config(model, config)
        o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
        o.set_field(x._abi.FIELD_U, model.momentum.U)
        o.set_field(x._abi.FIELD_P, model.momentum.p)
        res, _ = o.simple_iterate(4)
        out[grad] = (res, o.get_field(x._abi.FIELD_GRADP))
    assert np.all(np.isfinite(out["midpoint"][0]))
    assert not np.array_equal(out["gauss"][1], out["midpoint"][1])
