"""Meshes read from UNV files on the GPU against the oracle (1e-10 relative
L2, expected 0): the reference's hex cavity and tetrahedral streamtube
(3D, committed raw parses), SIMPLE host-polled and in graph mode."""
import numpy as np
import pytest

from test_unv3 import unv3_case, unv3_fixture_mesh

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("name", ["cavity_hex_unv3.npz", "streamtube_unv3.npz"])
def test_unv3_parity(x, orc, ctx, name, graph):
    mesh = unv3_fixture_mesh(x, name)
    model, config = unv3_case(x, mesh, 10)
    cfg, keep = x.build_config(model, config, pref=0.0 if name.startswith("cavity") else None)
    dm = x.DeviceMesh(ctx, mesh)
    g = x.Case(dm, cfg)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    for c in (g, o):
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
    if graph:
        g.set_graph_mode(True)
    rg, _ = g.simple_iterate(10)
    ro, _ = o.simple_iterate(10)
    assert rel(rg, ro) <= TOL, (rg, ro)
    for f in (x._abi.FIELD_U, x._abi.FIELD_P, x._abi.FIELD_MDOTF):
        assert rel(g.get_field(f), o.get_field(f)) <= TOL, f
