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
