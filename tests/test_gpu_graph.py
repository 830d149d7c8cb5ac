"""Graph mode: a SIMPLE iteration / PISO step replayed as one CUDA graph with
device-driven Krylov loops (conditional WHILE nodes) gives the same results,
bit for bit, as the default host-polled mode -- FP64 and mixed precision,
steady and transient (periodic LES)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(x, ctx, mesh, model, config, graph, steps, pref=None, piso=False):
    cfg, keep = x.build_config(model, config, pref=pref)
    dm = x.DeviceMesh(ctx, mesh)
    c = x.Case(dm, cfg)
    c.set_field(x._abi.FIELD_U, model.momentum.U)
    c.set_field(x._abi.FIELD_P, model.momentum.p)
    if graph:
        c.set_graph_mode(True)
    if piso:
        res, co = c.piso_step(steps)
    else:
        res, conv = c.simple_iterate(steps)
        co = None
    return res, co, c.get_field(x._abi.FIELD_U), c.get_field(x._abi.FIELD_P), (c, dm, keep)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_graph_simple_identical(x, ctx, prec):
    mesh = x.build_mesh3(x.channel_polymesh(16, 8, 8, seed=11))
    out = []
    for graph in (False, True):
        model, config = x.cases.channel_case(mesh, iterations=6, precision=prec)
        out.append(_run(x, ctx, mesh, model, config, graph, 6))
    (r0, _, U0, p0, _), (r1, _, U1, p1, _) = out
    assert np.array_equal(r0, r1), (r0, r1)
    assert np.array_equal(U0, U1) and np.array_equal(p0, p1)


def test_graph_cavity_dilu_identical(x, ctx):
    mesh = x.build_mesh3(x.cavity_polymesh(20))
    out = []
    for graph in (False, True):
        model, config = x.cases.cavity_case(mesh, iterations=10)
        out.append(_run(x, ctx, mesh, model, config, graph, 10, pref=0.0))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][2], out[1][2]) and np.array_equal(out[0][3], out[1][3])


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_graph_piso_periodic_identical(x, ctx, prec):
    mesh = x.build_mesh3(x.periodic_box_polymesh(10, seed=4))
    U0 = x.cases.fourier_field(mesh, seed=4)
    out = []
    for graph in (False, True):
        model, config = x.cases.periodic_les_case(mesh, steps=4, U0=U0, precision=prec)
        out.append(_run(x, ctx, mesh, model, config, graph, 4, pref=0.0, piso=True))
    (r0, c0, U0_, p0, _), (r1, c1, U1, p1, _) = out
    assert np.array_equal(r0, r1), (r0, r1)
    assert np.array_equal(c0, c1)
    assert np.array_equal(U0_, U1) and np.array_equal(p0, p1)


def test_graph_launch_count_reported(x, ctx):
    """Launch counting follows the kernels the WHILE bodies actually ran."""
    mesh = x.build_mesh3(x.channel_polymesh(12, 6, 6, seed=1))
    model, config = x.cases.channel_case(mesh, iterations=3)
    cfg, keep = x.build_config(model, config)
    dm = x.DeviceMesh(ctx, mesh)
    c = x.Case(dm, cfg)
    c.set_field(x._abi.FIELD_U, model.momentum.U)
    c.set_field(x._abi.FIELD_P, model.momentum.p)
    c.simple_iterate(1)
    c.set_graph_mode(True)
    l0 = x.launch_count()
    c.simple_iterate(2)
    n = x.launch_count() - l0
    assert n > 50, n


def test_autotuner_choices(x, ctx):
    """The autotuner picks a valid launch shape per equation; parity with the
    oracle under those shapes is covered by the SIMPLE parity tests (they run
    through simple_iterate, which tunes first)."""
    mesh = x.build_mesh3(x.channel_polymesh(24, 12, 12, seed=5))
    model, config = x.cases.channel_case(mesh, iterations=2)
    cfg, keep = x.build_config(model, config)
    dm = x.DeviceMesh(ctx, mesh)
    c = x.Case(dm, cfg)
    t = c.tuning()
    assert t["U"]["spmv_rows_per_thread"] in (0, 1, 2, 4)
    assert t["U"]["spmv_block"] in (128, 256, 512)
    assert isinstance(t["U"]["dilu_one_block"], bool)
    c.set_field(x._abi.FIELD_U, model.momentum.U)
    c.set_field(x._abi.FIELD_P, model.momentum.p)
    r1, _ = c.simple_iterate(2)
    # a second case of the same size class reuses the cached choices
    c2 = x.Case(x.DeviceMesh(ctx, mesh), cfg)
    assert c2.tuning() == t


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_persistent_cg_identical(x, ctx, prec):
    """The pressure CG as one launch (q on chip) gives the two-kernel loop's
    results bit for bit, in each form: the automatic choice, the cluster form
    (14 tiles: one 16-block cluster, hardware barriers), the 1024-, 512-
    and 256-thread cooperative forms forced, and the one-block-per-SM forms
    (here one tile per block)."""
    mesh = x.build_mesh3(x.channel_polymesh(48, 24, 24, seed=6))
    out = []
    modes = (False, True, 2, 1024, 512, 256, 4, 5)
    for persist in modes:
        model, config = x.cases.channel_case(mesh, iterations=4, precision=prec)
        cfg, keep = x.build_config(model, config)
        dm = x.DeviceMesh(ctx, mesh)
        c = x.Case(dm, cfg)
        c.set_persistent(persist)
        c.set_inner_cg(1)  # mixed: the canonical FP32 kernels in every form
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
        c.set_profiling(True)
        res, _ = c.simple_iterate(4)
        ms, its = c.profile(5)
        out.append((res, c.get_field(x._abi.FIELD_U), c.get_field(x._abi.FIELD_P), its))
    assert out[0][3] == 0                        # the persistent kernel ran only when enabled
    for m, o in zip(modes[1:], out[1:]):
        assert o[3] > 0, m
        assert np.array_equal(out[0][0], o[0]), m
        assert np.array_equal(out[0][1], o[1]) and np.array_equal(out[0][2], o[2]), m


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_persistent_multi_tile_identical(x, ctx, prec):
    """One block per SM owning several tiles (160 tiles over at most 148
    blocks: some blocks run two) gives the two-kernel loop's results bit for
    bit, with 1024 and with 512 threads per block."""
    mesh = x.build_mesh3(x.channel_polymesh(80, 64, 64, seed=9))
    assert mesh.n_cells > 148 * 2048
    out = []
    for persist in (False, 4, 5):
        model, config = x.cases.channel_case(mesh, iterations=2, precision=prec)
        cfg, keep = x.build_config(model, config)
        dm = x.DeviceMesh(ctx, mesh)
        c = x.Case(dm, cfg)
        c.set_persistent(persist)
        c.set_inner_cg(1)
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
        c.set_profiling(True)
        res, _ = c.simple_iterate(2)
        ms, its = c.profile(5)
        out.append((res, c.get_field(x._abi.FIELD_U), c.get_field(x._abi.FIELD_P), its))
        c.close()
        dm.close()
    assert out[0][3] == 0
    for o in out[1:]:
        assert o[3] > 0
        assert np.array_equal(out[0][0], o[0])
        assert np.array_equal(out[0][1], o[1]) and np.array_equal(out[0][2], o[2])
