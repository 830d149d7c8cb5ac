"""The reference's end-to-end cases with known answers, on the GPU against
the oracle (1e-10 relative L2, expected 0) and against the known answer:

* 2d_incompressible_pitzdaily_Smagorinsky.jl on its polyMesh (committed
  fixture): 100 PISO+LES steps, outlet Ux = 7.60 +- 0.1;
* 2d_incompressible_laminar_BFS.jl on its 2D UNV grid (committed raw parse):
  500 SIMPLE iterations with the Jacobi smoother, outlet Ux = 0.5 inlet Ux
  +- 0.05; the smoother also inside a batch (bit for bit as alone);
* the pitzDaily configuration on a generated slab channel (filter width
  (V/distance)^0.5, Extrapolated nut, absolute-tolerance solves),
  host-polled and in graph mode."""
import numpy as np
import pytest

from test_oracle_golden import _polymesh
from test_reference_cases import slab_channel, slab_les_case
from test_unv import bfs_case, bfs_mesh, check_bfs_answer

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


def _pair(x, ctx, orc, mesh, model, cfg, graph=False):
    g = x.Case(x.DeviceMesh(ctx, mesh), cfg)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    for c in (g, o):
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
    if graph:
        g.set_graph_mode(True)
    return g, o


@pytest.mark.parametrize("graph", [False, True])
def test_pitzdaily_known_answer_gpu(x, orc, ctx, graph):
    mesh = x.build_mesh3(_polymesh(x, "pitzdaily_polymesh.npz"))
    assert mesh.n_cells == 12225
    model, config = slab_les_case(x, mesh, 100, 1e-5)
    cfg, keep = x.build_config(model, config, inner_loops=2)
    g, o = _pair(x, ctx, orc, mesh, model, cfg, graph)
    rg, _ = g.piso_step(100)
    ro, _ = o.piso_step(100)
    assert rel(rg, ro) <= TOL
    for f in (x._abi.FIELD_U, x._abi.FIELD_P, x._abi.FIELD_NUT):
        assert rel(g.get_field(f), o.get_field(f)) <= TOL, f
    U = g.get_field(x._abi.FIELD_U)
    outlet = x.api.boundary_average("outlet", U, config.boundaries["U"], mesh=mesh)
    assert abs(outlet[0] - 7.60) <= 0.1, outlet


@pytest.mark.parametrize("graph", [False, True])
def test_bfs_known_answer_gpu(x, orc, ctx, graph):
    mesh = bfs_mesh(x)
    model, config = bfs_case(x, mesh)
    cfg, keep = x.build_config(model, config)
    g, o = _pair(x, ctx, orc, mesh, model, cfg, graph)
    rg, _ = g.simple_iterate(500)
    ro, _ = o.simple_iterate(500)
    assert rel(rg, ro) <= TOL
    for f in (x._abi.FIELD_U, x._abi.FIELD_P):
        assert rel(g.get_field(f), o.get_field(f)) <= TOL, f
    check_bfs_answer(x, g.get_field(x._abi.FIELD_U), config, mesh)


def test_smoother_in_batch(x, ctx):
    """Two BFS cases, with and without the smoother, in one batch: each as alone."""
    mesh = bfs_mesh(x)
    iters = 20

    def mk(sm):
        model, config = bfs_case(x, mesh, iterations=iters, smoother=sm)
        cfg, keep = x.build_config(model, config)
        dm = x.DeviceMesh(ctx, mesh)
        c = x.Case(dm, cfg)
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
        return c, (dm, keep)

    alone = []
    for sm in (True, False):
        c, keep = mk(sm)
        res, _ = c.simple_iterate(iters)
        alone.append((res, c.get_field(x._abi.FIELD_U)))
    assert not np.array_equal(alone[0][1], alone[1][1])
    batch = x.api.Batch(ctx, 4, 1 << 32)
    members = [mk(sm) for sm in (True, False)]
    for c, _ in members:
        assert batch.add(c)
    hist = np.stack([batch.simple_iterate()[0] for _ in range(iters)], axis=1)
    for k, (c, _) in enumerate(members):
        assert np.array_equal(hist[k], alone[k][0]), k
        assert np.array_equal(c.get_field(x._abi.FIELD_U), alone[k][1]), k
    batch.close()
