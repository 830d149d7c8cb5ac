"""A mesh that arrives as an OpenFOAM polyMesh directory (written, then read
back by FOAM3D_mesh) runs the SIMPLE path on the GPU with the oracle's
results: a 3D lid-driven cube with the reference grid's patch names
("walls" on five sides, the moving "top"), permuted numbering.

Tolerance: the 1e-10 relative L2 of the FP64 parity tests (expected 0)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


def test_polymesh_cube_simple_parity(x, orc, ctx, tmp_path):
    pm = x.box_polymesh(10, 9, 8, lengths=(1.0, 1.0, 1.0),
                        patches=[("walls", ["xmin", "xmax", "ymin", "zmin", "zmax"]), ("top", ["ymax"])], seed=12)
    d = str(tmp_path / "polyMesh")
    x.write_polymesh(pm, d)
    mesh = x.FOAM3D_mesh(d)
    A = x.api
    model = A.Physics(time=A.Steady(), fluid=A.Fluid(A.Incompressible, nu=0.01), turbulence=A.RANS(A.Laminar),
                      energy=A.Energy(A.Isothermal), domain=mesh)
    BCs = A.assign(region=mesh, U=[A.Wall("walls", [0.0, 0.0, 0.0]), A.Wall("top", [1.0, 0.0, 0.0])],
                   p=[A.Wall("walls"), A.Wall("top")])
    solvers = {"U": A.SolverSetup(solver=A.Bicgstab(), preconditioner=A.DILU(), convergence=1e-7, relax=0.7),
               "p": A.SolverSetup(solver=A.Cg(), preconditioner=A.Jacobi(), convergence=1e-7, relax=0.3)}
    config = A.Configuration(solvers=solvers, schemes={"U": A.Schemes(divergence=A.Upwind), "p": A.Schemes()},
                             runtime=A.Runtime(iterations=5, write_interval=-1, time_step=1.0),
                             hardware=A.Hardware(backend=A.B200Backend()), boundaries=BCs)
    A.initialise_(model.momentum.U, [0.0, 0.0, 0.0])
    A.initialise_(model.momentum.p, 0.0)
    cfg, keep = x.build_config(model, config, pref=0.0)
    dm = x.DeviceMesh(ctx, mesh)
    g = x.Case(dm, cfg)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    for c in (g, o):
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
    rg, _ = g.simple_iterate(5)
    ro, _ = o.simple_iterate(5)
    assert rel(rg, ro) <= TOL, (rg, ro)
    for f in (x._abi.FIELD_U, x._abi.FIELD_P):
        assert rel(g.get_field(f), o.get_field(f)) <= TOL
