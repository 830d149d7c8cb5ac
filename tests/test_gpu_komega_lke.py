"""RANS{KOmegaLKE} on the GPU against the oracle (1e-10 relative L2,
expected 0): the flat plate of examples/2D_flatplate_LKE_ERCOFTAC.jl (steady
SIMPLE, OmegaWallFunction on the wall) host-polled with Jacobi and DILU and
in graph mode; the wall distance; a restart from a checkpoint; LKE cases in
a batch equal to the same cases alone; run_ writing k, omega, kl, nut and y."""
import os

import numpy as np
import pytest

from test_komega_lke import KL_FIELDS, flatplate, set_lke_fields

pytestmark = pytest.mark.gpu

TOL = 1e-10
ALL = KL_FIELDS + ("FIELD_GAMMA", "FIELD_NUTF", "FIELD_NUEFF", "FIELD_GRADU", "FIELD_PK", "FIELD_DK", "FIELD_DW")


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


def _pair(x, orc, ctx, mesh, model, cfg, graph=False):
    dm = x.DeviceMesh(ctx, mesh)
    g = x.Case(dm, cfg)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    for c in (g, o):
        set_lke_fields(x, c, model)
    if graph:
        g.set_graph_mode(True)
    return g, o, dm


@pytest.mark.parametrize("precond,graph", [("Jacobi", False), ("DILU", False), ("Jacobi", True)])
def test_lke_flatplate_parity(x, orc, ctx, precond, graph):
    mesh = flatplate(x, 30, 14, seed=5)
    model, config = x.cases.lke_flatplate_case(mesh, 12, precond=getattr(x.api, precond))
    cfg, keep = x.build_config(model, config)
    g, o, dm = _pair(x, orc, ctx, mesh, model, cfg, graph)
    assert rel(g.get_field(x._abi.FIELD_WALLDIST), o.get_field(x._abi.FIELD_WALLDIST)) <= TOL
    rg, _ = g.simple_iterate(12)
    ro, _ = o.simple_iterate(12)
    assert rel(rg, ro) <= TOL, (rg, ro)
    for f in ALL:
        assert rel(g.get_field(getattr(x._abi, f)), o.get_field(getattr(x._abi, f))) <= TOL, f


def test_lke_restart_bit_identical(x, ctx):
    """checkpoint() / restore() carry kl too: 3 + 3 iterations from a
    restored case equal 6 in one go."""
    mesh = flatplate(x, 20, 10)

    def new_case():
        model, config = x.cases.lke_flatplate_case(mesh, 6)
        cfg, keep = x.build_config(model, config)
        dm = x.DeviceMesh(ctx, mesh)
        c = x.Case(dm, cfg)
        set_lke_fields(x, c, model)
        return c, (dm, keep)

    a, ka = new_case()
    ra = a.simple_iterate(6)[0]
    b, kb = new_case()
    rb = b.simple_iterate(3)[0]
    state = b.checkpoint()
    assert "FIELD_KL" in state
    c, kc = new_case()
    c.restore(state)
    rc = c.simple_iterate(3)[0]
    assert np.array_equal(np.concatenate([rb, rc]), ra)
    for f in KL_FIELDS:
        assert np.array_equal(c.get_field(getattr(x._abi, f)), a.get_field(getattr(x._abi, f))), f


def test_lke_batch_matches_single(x, ctx):
    """LKE cases in a batch (their U and p solves batched, kl / omega / k on
    each case's stream) equal the same cases advanced alone, bit for bit."""
    specs = [(24, 12, 1), (20, 10, 2)]

    def mk(nx, ny, seed):
        mesh = flatplate(x, nx, ny, seed)
        model, config = x.cases.lke_flatplate_case(mesh, 4)
        cfg, keep = x.build_config(model, config)
        dm = x.DeviceMesh(ctx, mesh)
        c = x.Case(dm, cfg)
        c.set_inner_cg(1)
        set_lke_fields(x, c, model)
        return c, (dm, keep, cfg)

    alone = []
    for s in specs:
        c, keep = mk(*s)
        res, _ = c.simple_iterate(4)
        alone.append((res, [c.get_field(getattr(x._abi, f)) for f in KL_FIELDS]))
    batch = x.api.Batch(ctx, 4, 1 << 32)
    members = []
    for s in specs:
        c, keep = mk(*s)
        assert batch.add(c)
        members.append((c, keep))
    hist = np.stack([batch.simple_iterate()[0] for _ in range(4)], axis=1)
    for k, (c, keep) in enumerate(members):
        assert np.array_equal(hist[k], alone[k][0]), k
        for f, ref in zip(KL_FIELDS, alone[k][1]):
            assert np.array_equal(c.get_field(getattr(x._abi, f)), ref), (k, f)
    batch.close()


def test_lke_run_writes_fields(x, tmp_path):
    """run_ through the public API: the model's k, omega, kl, nut and y come
    back from the device; the VTK file carries them (save_output,
    RANS_kOmegaLKE.jl:478-489)."""
    mesh = flatplate(x, 20, 10)
    model, config = x.cases.lke_flatplate_case(mesh, 5)
    config.runtime.write_interval = 5
    x.api.run_(model, config, output_dir=str(tmp_path))
    t = model.turbulence
    for v in (t.k, t.omega, t.kl, t.nut, t.y):
        assert np.all(np.isfinite(v)) and v.max() > 0.0
    files = sorted(os.listdir(tmp_path))
    assert files, files
    text = open(os.path.join(tmp_path, files[-1])).read()
    for name in ("\"k\"", "\"omega\"", "\"kl\"", "\"nut\"", "\"y\""):
        assert name in text, name


def test_lke_mixed_precision(x, ctx):
    """Mixed precision (FP32 inner solves of U, p, kl, omega and k inside the
    FP64 defect correction): after 12 SIMPLE iterations every field is within
    1e-3 relative L2 of the FP64 run.  The iterations' solves stop at rtol
    0.01 (p 1e-3), so the two runs differ at that level until convergence
    (measured: U 4e-7, p 1.4e-4, k 1.2e-4, omega 5e-5, kl 2e-5, nut 8e-5)."""
    mesh = flatplate(x, 30, 14, seed=5)
    out = {}
    for prec in ("fp64", "mixed"):
        model, config = x.cases.lke_flatplate_case(mesh, 12, precision=prec)
        cfg, keep = x.build_config(model, config)
        dm = x.DeviceMesh(ctx, mesh)
        c = x.Case(dm, cfg)
        set_lke_fields(x, c, model)
        c.simple_iterate(12)
        out[prec] = {f: c.get_field(getattr(x._abi, f)) for f in KL_FIELDS}
        c.close()
        dm.close()
    for f in KL_FIELDS:
        assert rel(out["mixed"][f], out["fp64"][f]) <= 1e-3, f


def test_lke_dilu_scalars_jacobi_p_parity(x, orc, ctx):
    """kl, omega and k DILU-preconditioned while p is Jacobi (the p system's
    storage carries their DILU levels): GPU equal to the oracle."""
    mesh = flatplate(x, 30, 14, seed=5)
    model, config = x.cases.lke_flatplate_case(mesh, 8, precond=x.api.DILU)
    A = x.api
    config.solvers["p"] = A.SolverSetup(solver=A.Cg(), preconditioner=A.Jacobi(), convergence=1e-8, relax=0.2,
                                        rtol=1e-3)
    cfg, keep = x.build_config(model, config)
    assert cfg.p_solver.precond == x._abi.PRECOND_JACOBI and cfg.kl_solver.precond == x._abi.PRECOND_DILU
    g, o, dm = _pair(x, orc, ctx, mesh, model, cfg)
    rg, _ = g.simple_iterate(8)
    ro, _ = o.simple_iterate(8)
    assert rel(rg, ro) <= TOL, (rg, ro)
    for f in ALL:
        assert rel(g.get_field(getattr(x._abi, f)), o.get_field(getattr(x._abi, f))) <= TOL, f


def test_lke_periodic_channel_parity(x, orc, ctx):
    """k-omega LKE on a channel periodic in the flow direction (inlet and
    outlet paired by construct_periodic; U, p, k, kl, omega and nut periodic
    there) with a disturbed initial velocity: kl's periodic pairs in the
    shared p storage as k's and omega's; GPU equal to the oracle over 3
    SIMPLE iterations."""
    A = x.api
    mesh = x.build_mesh3(x.channel_polymesh(12, 6, 6, seed=7))
    per = list(A.construct_periodic(mesh, None, "inlet", "outlet"))
    model = A.Physics(time=A.Steady(), fluid=A.Fluid(A.Incompressible, nu=1e-3),
                      turbulence=A.RANS(A.KOmegaLKE, Tu=0.02, walls=["walls"]), energy=A.Energy(A.Isothermal),
                      domain=mesh)
    BCs = A.assign(region=mesh, U=per + [A.Wall("walls", [0.0, 0.0, 0.0])], p=per + [A.Wall("walls")],
                   k=per + [A.Dirichlet("walls", 0.0)], kl=per + [A.Dirichlet("walls", 0.0)],
                   omega=per + [A.OmegaWallFunction("walls")], nut=per + [A.Dirichlet("walls", 0.0)])

    def ss(s, relax):
        return A.SolverSetup(solver=s(), preconditioner=A.Jacobi(), convergence=1e-7, relax=relax, rtol=1e-2)

    config = A.Configuration(solvers={"U": ss(A.Bicgstab, 0.7), "p": ss(A.Cg, 0.3), "k": ss(A.Bicgstab, 0.5),
                                      "kl": ss(A.Bicgstab, 0.5), "omega": ss(A.Bicgstab, 0.5),
                                      "y": A.SolverSetup(solver=A.Cg(), preconditioner=A.Jacobi(), convergence=1e-8,
                                                         relax=0.9, rtol=1e-3)},
                             schemes={"U": A.Schemes(divergence=A.Upwind), "p": A.Schemes(),
                                      "k": A.Schemes(divergence=A.Upwind), "kl": A.Schemes(divergence=A.Upwind),
                                      "omega": A.Schemes(divergence=A.Upwind), "y": A.Schemes()},
                             runtime=A.Runtime(iterations=3, write_interval=-1, time_step=1.0),
                             hardware=A.Hardware(backend=A.B200Backend()), boundaries=BCs)
    rng = np.random.default_rng(7)
    model.momentum.U[:] = np.array([[1.0], [0.0], [0.0]]) + 0.05 * rng.standard_normal((3, mesh.n_cells))
    A.initialise_(model.momentum.p, 0.0)
    A.initialise_(model.turbulence.k, 0.01)
    A.initialise_(model.turbulence.kl, 0.005)
    A.initialise_(model.turbulence.omega, 10.0)
    A.initialise_(model.turbulence.nut, 1e-3)
    cfg, keep = x.build_config(model, config, pref=0.0)
    g, o, dm = _pair(x, orc, ctx, mesh, model, cfg)
    rg, _ = g.simple_iterate(3)
    ro, _ = o.simple_iterate(3)
    assert rel(rg, ro) <= TOL, (rg, ro)
    for f in ALL:
        assert rel(g.get_field(getattr(x._abi, f)), o.get_field(getattr(x._abi, f))) <= TOL, f
