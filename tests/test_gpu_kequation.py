"""LES{KEquation} on the GPU against the oracle (tolerance 0): a channel with
a disturbed inflow, PISO steps with the subgrid k equation, host-polled and
in graph mode -- U, p, k, nut, their face values, grad U and the k
equation's sources equal bit for bit; a checkpoint/restore continues
exactly; mixed precision stays within the mixed-precision tolerance; the
batch (steady SIMPLE only) refuses the transient model."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("FIELD_U", "FIELD_P", "FIELD_K", "FIELD_NUT", "FIELD_NUTF", "FIELD_NUEFF", "FIELD_GRADU", "FIELD_PK",
          "FIELD_DK", "FIELD_DW")


def _set(x, c, model):
    A = x._abi
    for f, v in (("FIELD_U", model.momentum.U), ("FIELD_P", model.momentum.p), ("FIELD_K", model.turbulence.k),
                 ("FIELD_NUT", model.turbulence.nut)):
        c.set_field(getattr(A, f), v)


def _gpu(x, ctx, mesh, model, cfg, graph=False):
    dm = x.DeviceMesh(ctx, mesh)
    g = x.Case(dm, cfg)
    _set(x, g, model)
    if graph:
        g.set_graph_mode(True)
    return g, dm


@pytest.mark.parametrize("graph", [False, True])
def test_kequation_parity(x, orc, ctx, graph):
    mesh = x.build_mesh3(x.channel_polymesh(24, 10, 10, seed=5))
    model, config = x.cases.kequation_channel_case(mesh, steps=6)
    cfg, keep = x.build_config(model, config)
    g, dm = _gpu(x, ctx, mesh, model, cfg, graph)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    _set(x, o, model)
    rg, cg = g.piso_step(6)
    ro, co = o.piso_step(6)
    assert np.array_equal(rg, ro) and np.array_equal(cg, co)
    for f in FIELDS:
        a, b = g.get_field(getattr(x._abi, f)), o.get_field(getattr(x._abi, f))
        assert np.array_equal(a, b), f
    assert g.get_field(x._abi.FIELD_K).max() > 0.0


def test_kequation_restart_and_mixed(x, ctx):
    mesh = x.build_mesh3(x.channel_polymesh(24, 10, 10, seed=5))
    model, config = x.cases.kequation_channel_case(mesh, steps=6)
    cfg, keep = x.build_config(model, config)
    a, dma = _gpu(x, ctx, mesh, model, cfg)
    ra, _ = a.piso_step(6)
    b, dmb = _gpu(x, ctx, mesh, model, cfg)
    b.piso_step(3)
    state = b.checkpoint()
    assert "FIELD_K" in state
    c, dmc = _gpu(x, ctx, mesh, model, cfg)
    c.restore(state)
    rc, _ = c.piso_step(3)
    assert np.array_equal(rc, ra[3:])
    for f in ("FIELD_U", "FIELD_P", "FIELD_K", "FIELD_NUT"):
        assert np.array_equal(c.get_field(getattr(x._abi, f)), a.get_field(getattr(x._abi, f))), f
    # mixed precision: FP32 inner solves, same fields within the tolerance
    mm, mc = x.cases.kequation_channel_case(mesh, steps=6, precision="mixed")
    cfg_m, keep_m = x.build_config(mm, mc)
    m, dmm = _gpu(x, ctx, mesh, mm, cfg_m)
    m.piso_step(6)
    for f in ("FIELD_U", "FIELD_K", "FIELD_NUT"):
        ref = a.get_field(getattr(x._abi, f))
        err = np.linalg.norm(m.get_field(getattr(x._abi, f)) - ref) / np.linalg.norm(ref)
        assert err <= 1e-4, (f, err)


@pytest.mark.parametrize("graph", [False, True])
def test_kequation_periodic_parity(x, orc, ctx, graph):
    """The periodic LES box with the k equation: k's periodic pairs in the
    shared p storage, GPU equal to the oracle bit for bit over 4 steps."""
    mesh = x.build_mesh3(x.periodic_box_polymesh(10, seed=4))
    U0 = x.cases.fourier_field(mesh, seed=4)
    model, config = x.cases.periodic_les_case(mesh, steps=4, U0=U0, model_kind=x.KEquation)
    cfg, keep = x.build_config(model, config)
    assert cfg.turbulence == x._abi.TURB_KEQUATION
    g, dm = _gpu(x, ctx, mesh, model, cfg, graph)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    _set(x, o, model)
    rg, cg = g.piso_step(4)
    ro, co = o.piso_step(4)
    assert np.array_equal(rg, ro) and np.array_equal(cg, co)
    for f in FIELDS:
        a, b = g.get_field(getattr(x._abi, f)), o.get_field(getattr(x._abi, f))
        assert np.array_equal(a, b), f


def test_kequation_batch_refused(x, ctx):
    mesh = x.build_mesh3(x.channel_polymesh(12, 6, 6, seed=1))
    model, config = x.cases.kequation_channel_case(mesh, steps=2)
    cfg, keep = x.build_config(model, config)
    g, dm = _gpu(x, ctx, mesh, model, cfg)
    batch = x.api.Batch(ctx, 4, 1 << 30)
    with pytest.raises(Exception):
        batch.add(g)
    batch.close()
