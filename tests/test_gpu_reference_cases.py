"""The pitzDaily Smagorinsky configuration (2D slab with Empty front/back:
filter width (V/distance)^0.5, Extrapolated nut at inlet and outlet,
Jacobi-preconditioned solves to an absolute tolerance) on a generated slab
channel: GPU against the oracle (1e-10 relative L2, expected 0), host-polled
and in graph mode."""
import numpy as np
import pytest

from test_reference_cases import slab_channel, slab_les_case

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("graph", [False, True])
def test_slab_les_parity(x, orc, ctx, graph):
    mesh = slab_channel(x, nx=40, ny=12, seed=5)
    model, config = slab_les_case(x, mesh, 6, 2e-3, U_inlet=1.0, nu=1e-4)
    cfg, keep = x.build_config(model, config, inner_loops=2)
    assert cfg.les_delta_power == 0.5
    dm = x.DeviceMesh(ctx, mesh)
    g = x.Case(dm, cfg)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    for c in (g, o):
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
    if graph:
        g.set_graph_mode(True)
    rg, _ = g.piso_step(6)
    ro, _ = o.piso_step(6)
    assert rel(rg, ro) <= TOL, (rg, ro)
    for f in (x._abi.FIELD_U, x._abi.FIELD_P, x._abi.FIELD_NUT, x._abi.FIELD_DELTA, x._abi.FIELD_NUEFF):
        assert rel(g.get_field(f), o.get_field(f)) <= TOL, f
    U = g.get_field(x._abi.FIELD_U)
    assert x.api.boundary_average("inlet", U, config.boundaries["U"], mesh=mesh)[0] == pytest.approx(1.0)
