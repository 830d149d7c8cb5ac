"""The reference's own end-to-end case with a known answer, on the CPU
oracle: test/0_TEST_CASES/2d_incompressible_pitzdaily_Smagorinsky.jl
(pitzDaily polyMesh read in place where the reference checkout is present:
12225 cells / 49180 faces / 25012 nodes; PISO + Smagorinsky, 100 steps of
1e-5 s, inner_loops 2; the test expects the inlet average Ux = 10 and the
outlet average Ux = 7.60 +- 0.1).  Also the LES filter scaling of such a 2D
slab (delta_scaling, LES_functions.jl:33-56) and boundary_average
(Postprocess_functions.jl:157-185)."""
import os

import numpy as np
import pytest
from refpath import ref_path

PITZ = ref_path("examples/0_GRIDS/OF_pitzDaily/polyMesh")


def slab_les_case(x, mesh, steps, dt, U_inlet=10.0, nu=1e-5, walls=("upperWall", "lowerWall")):
    """The pitzDaily Smagorinsky configuration (2d_incompressible_pitzdaily_
    Smagorinsky.jl:31-116) on a mesh with patches inlet, outlet, the walls
    and frontAndBack (Empty)."""
    A = x.api
    model = A.Physics(time=A.Transient(), fluid=A.Fluid(A.Incompressible, nu=nu), turbulence=A.LES(A.Smagorinsky),
                      energy=A.Energy(A.Isothermal), domain=mesh)
    BCs = A.assign(region=mesh,
                   U=[A.Dirichlet("inlet", [U_inlet, 0.0, 0.0]), A.Zerogradient("outlet"), A.Empty("frontAndBack")]
                   + [A.Wall(w, [0.0, 0.0, 0.0]) for w in walls],
                   p=[A.Zerogradient("inlet"), A.Dirichlet("outlet", 0.0), A.Empty("frontAndBack")]
                   + [A.Wall(w, 0.0) for w in walls],
                   nut=[A.Extrapolated("inlet"), A.Extrapolated("outlet", 0.0), A.Empty("frontAndBack")]
                   + [A.Dirichlet(w, 0.0) for w in walls])
    solvers = {k: A.SolverSetup(solver=s(), preconditioner=A.Jacobi(), convergence=1e-7, atol=1e-5, rtol=0.0, relax=1.0)
               for k, s in (("U", A.Bicgstab), ("p", A.Cg))}
    schemes = {"U": A.Schemes(time=A.Euler, divergence=A.Upwind, gradient=A.Gauss),
               "p": A.Schemes(time=A.Euler, divergence=A.Upwind, gradient=A.Gauss)}
    config = A.Configuration(solvers=solvers, schemes=schemes,
                             runtime=A.Runtime(iterations=steps, time_step=dt, write_interval=steps),
                             hardware=A.Hardware(backend=A.B200Backend()), boundaries=BCs)
    A.initialise_(model.momentum.U, [0.0, 0.0, 0.0])
    A.initialise_(model.momentum.p, 0.0)
    return model, config


def slab_channel(x, nx=24, ny=8, seed=2):
    """A 2D channel slab: [0, 2] x [0, 0.5] x [0, 0.05], one cell thick."""
    pm = x.box_polymesh(nx, ny, 1, lengths=(2.0, 0.5, 0.05), seed=seed,
                        patches=[("inlet", ["xmin"]), ("outlet", ["xmax"]), ("upperWall", ["ymax"]),
                                 ("lowerWall", ["ymin"]), ("frontAndBack", ["zmin", "zmax"])])
    return x.build_mesh3(pm)


def test_delta_scaling_and_boundary_average(x):
    mesh = slab_channel(x)
    A = x.api
    model, config = slab_les_case(x, mesh, 1, 1e-3)
    # Empty patches at z = 0 and z = 0.05: distance 0.05, power 0.5
    d, pw = A.delta_scaling(mesh, config.boundaries["U"])
    assert pw == 0.5 and abs(d - 0.05) < 1e-15
    assert A.delta_scaling(mesh, [A.Wall("upperWall")]) == (1.0, 1.0 / 3.0)
    U = np.zeros((3, mesh.n_cells))
    U[0] = np.arange(mesh.n_cells, dtype=np.float64)
    bcs = config.boundaries["U"]
    assert np.array_equal(A.boundary_average("inlet", U, bcs, mesh=mesh), [10.0, 0.0, 0.0])
    out = A.boundary_average("outlet", U, bcs, mesh=mesh)
    cells = np.asarray(mesh.boundary_cellsID)[list(mesh.patch_range("outlet"))]
    assert out[0] == pytest.approx(U[0, cells].mean(), rel=1e-15)
    assert np.array_equal(A.boundary_average("frontAndBack", U, bcs, mesh=mesh), [0.0, 0.0, 0.0])
    assert A.boundary_average("outlet", U[0], config.boundaries["p"], mesh=mesh) == 0.0


@pytest.mark.skipif(not os.path.isdir(PITZ), reason="XCAL_REFERENCE_DIR (an XCALibre.jl checkout) not set")
def test_pitzdaily_smagorinsky_known_answer(x, orc):
    mesh = x.FOAM3D_mesh(PITZ)
    assert (mesh.n_cells, mesh.n_faces, mesh.points.shape[0]) == (12225, 49180, 25012)
    model, config = slab_les_case(x, mesh, 100, 1e-5)
    cfg, keep = x.build_config(model, config, inner_loops=2, ncorrectors=0)
    assert cfg.les_delta_power == 0.5 and cfg.les_delta_distance > 0.0
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    o.set_field(x._abi.FIELD_U, model.momentum.U)
    o.set_field(x._abi.FIELD_P, model.momentum.p)
    res, _ = o.piso_step(100)
    assert res.shape == (100, 4) and np.all(np.isfinite(res))
    U = o.get_field(x._abi.FIELD_U)
    inlet = x.api.boundary_average("inlet", U, config.boundaries["U"], mesh=mesh)
    outlet = x.api.boundary_average("outlet", U, config.boundaries["U"], mesh=mesh)
    assert inlet[0] == pytest.approx(10.0)
    assert abs(outlet[0] - 7.60) <= 0.1, outlet
