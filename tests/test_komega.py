"""RANS{KOmega} (RANS_kOmega.jl) on the CPU oracle.

* the reference's known answer of
  test/0_TEST_CASES/2d_incompressible_transient_KOmega_BFS_lowRe.jl on its own
  grid (backwardFacingStep_5mm.unv, committed raw parse): 500 PISO steps of
  0.01 s with k and omega transported (OmegaWallFunction on the wall and top,
  Midpoint gradients), outlet Ux = 0.5 inlet Ux within 0.1 Umag;
* the wall-function constants (y_plus_laminar, RANS_functions.jl:42-45), the
  omega wall rows (constrain!, :376-429) and bound! (:2-41) on a few steps;
* the k and nut wall functions in the log layer (nutf = nut_wall(nu, y+));
* k-omega SST on a channel: the wall distance and a few SIMPLE iterations."""
import math
import os

import numpy as np
import pytest

from test_unv import bfs_mesh
from refpath import ref_path

REF = ref_path("examples/0_GRIDS/backwardFacingStep_5mm.unv")


def komega_bfs_case(x, mesh, steps=500, precision="fp64"):
    """2d_incompressible_transient_KOmega_BFS_lowRe.jl:11-121."""
    A = x.api
    nu, Umag, k_in, w_in = 1e-3, 1.5, 1.0, 1000.0
    model = A.Physics(time=A.Transient(), fluid=A.Fluid(A.Incompressible, nu=nu), turbulence=A.RANS(A.KOmega),
                      energy=A.Energy(A.Isothermal), domain=mesh)
    BCs = A.assign(region=mesh,
                   U=[A.Dirichlet("inlet", [Umag, 0.0, 0.0]), A.Extrapolated("outlet"),
                      A.Wall("wall", [0.0, 0.0, 0.0]), A.Dirichlet("top", [0.0, 0.0, 0.0])],
                   p=[A.Extrapolated("inlet"), A.Dirichlet("outlet", 0.0), A.Extrapolated("wall"),
                      A.Extrapolated("top")],
                   k=[A.Dirichlet("inlet", k_in), A.Extrapolated("outlet"), A.Dirichlet("wall", 0.0),
                      A.Dirichlet("top", 0.0)],
                   omega=[A.Dirichlet("inlet", w_in), A.Extrapolated("outlet"), A.OmegaWallFunction("wall"),
                          A.OmegaWallFunction("top")],
                   nut=[A.Dirichlet("inlet", k_in / w_in), A.Extrapolated("outlet"), A.Dirichlet("wall", 0.0),
                        A.Dirichlet("top", 0.0)])

    def sch():
        return A.Schemes(gradient=A.Midpoint, time=A.Euler)

    def ss(s):
        return A.SolverSetup(solver=s(), preconditioner=A.Jacobi(), convergence=1e-7, relax=1.0, rtol=1e-3)

    config = A.Configuration(solvers={"U": ss(A.Bicgstab), "p": ss(A.Cg), "k": ss(A.Bicgstab),
                                      "omega": ss(A.Bicgstab)},
                             schemes={"U": sch(), "p": A.Schemes(gradient=A.Midpoint), "k": sch(), "omega": sch()},
                             runtime=A.Runtime(iterations=steps, write_interval=steps, time_step=0.01),
                             hardware=A.Hardware(backend=A.B200Backend(precision=precision)), boundaries=BCs)
    A.initialise_(model.momentum.U, [Umag, 0.0, 0.0])
    A.initialise_(model.momentum.p, 0.0)
    A.initialise_(model.turbulence.k, k_in)
    A.initialise_(model.turbulence.omega, w_in)
    A.initialise_(model.turbulence.nut, k_in / w_in)
    return model, config


KW_FIELDS = ("FIELD_U", "FIELD_P", "FIELD_K", "FIELD_OMEGA", "FIELD_NUT")


def set_komega_fields(x, c, model):
    for f, v in (("FIELD_U", model.momentum.U), ("FIELD_P", model.momentum.p), ("FIELD_K", model.turbulence.k),
                 ("FIELD_OMEGA", model.turbulence.omega), ("FIELD_NUT", model.turbulence.nut)):
        c.set_field(getattr(x._abi, f), v)


@pytest.mark.skipif(not os.path.isfile(REF), reason="XCAL_REFERENCE_DIR (an XCALibre.jl checkout) not set")
def test_bfs_5mm_fixture_matches_file(x):
    a = x.UNV2D_mesh(REF, scale=0.001)
    b = bfs_mesh(x, 5)
    assert (a.n_cells, a.n_faces) == (7200, 14640)
    for k in ("face_owner", "face_neigh", "face_centre", "face_normal", "face_area", "face_delta", "face_weight",
              "cell_centre", "cell_volume", "cell_faces", "cell_nsign", "boundary_cellsID", "patch_start"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_komega_bfs_known_answer(x, orc):
    mesh = bfs_mesh(x, 5)
    model, config = komega_bfs_case(x, mesh)
    cfg, keep = x.build_config(model, config)
    assert cfg.turbulence == x._abi.TURB_KOMEGA and cfg.n_bc_omega == 4
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    set_komega_fields(x, o, model)
    res, _ = o.piso_step(500)
    assert np.all(np.isfinite(res))
    U = o.get_field(x._abi.FIELD_U)
    inlet = x.api.boundary_average("inlet", U, config.boundaries["U"], mesh=mesh)
    outlet = x.api.boundary_average("outlet", U, config.boundaries["U"], mesh=mesh)
    assert inlet[0] == pytest.approx(1.5)
    assert np.linalg.norm(outlet - 0.5 * inlet) <= 0.1 * 1.5, (inlet, outlet)
    k, w, nut = (o.get_field(getattr(x._abi, f)) for f in ("FIELD_K", "FIELD_OMEGA", "FIELD_NUT"))
    eps = np.spacing(1.0)
    assert k.min() >= eps and w.min() >= eps  # bound!
    assert np.array_equal(nut, k / w)


def test_komega_wall_rows(x, orc):
    """After a few steps every wall cell holds omega_vis or omega_log of the
    k it saw, and the constants are the reference's."""
    A = x.api
    bc = A.OmegaWallFunction("wall")
    yl = 11.0
    for _ in range(10):
        yl = math.log(max(yl * 9.8, 1.0)) / 0.41
    assert bc.wall == (0.41, 0.075, 0.09 ** 0.25, yl, 9.8)
    assert 11.0 < yl < 12.0
    mesh = bfs_mesh(x, 5)
    model, config = komega_bfs_case(x, mesh, steps=3)
    cfg, keep = x.build_config(model, config)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    set_komega_fields(x, o, model)
    o.piso_step(2)
    k_before = o.get_field(x._abi.FIELD_K)
    o.piso_step(1)
    w = o.get_field(x._abi.FIELD_OMEGA)
    # the last wall face of each cell (BC order wall, top; face order) sets its row
    last = {}
    for name in ("wall", "top"):
        for f in mesh.patch_range(name):
            last[int(mesh.boundary_cellsID[f])] = f
    nu = 1e-3
    for c, f in last.items():
        y = mesh.face_delta[f]
        sk = math.sqrt(k_before[c])
        w_vis = (6.0 * nu) / (0.075 * (y * y))
        w_log = sk / ((0.09 ** 0.25 * 0.41) * y)
        yplus = ((0.09 ** 0.25 * y) * sk) / nu
        expect = w_log if yplus > yl else w_vis
        assert w[c] == max(expect, np.spacing(1.0)), (c, w[c], expect)


def test_wall_function_values(x, orc):
    """NutWallFunction faces hold nut_wall(nu, y+) of their cell's k
    (RANS_functions.jl:61-63, 135-172) and KWallFunction keeps k finite:
    a k-omega channel at nu = 1e-5 (wall cells in the log layer), oracle."""
    from test_gpu_komega import komega_channel_case
    from test_nonorth_oracle import skewed_channel
    mesh = skewed_channel(x, n=(10, 6, 5), seed=5)
    model, config = komega_channel_case(x, mesh, 4, wallfn=True)
    cfg, keep = x.build_config(model, config)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    set_komega_fields(x, o, model)
    res, _ = o.simple_iterate(4)
    assert np.all(np.isfinite(res))
    k = o.get_field(x._abi.FIELD_K)
    nutf = o.get_field(x._abi.FIELD_NUTF)
    kappa, E, c25 = 0.41, 9.8, 0.09 ** 0.25
    yl = x.api.y_plus_laminar(E, kappa)
    for f in mesh.patch_range("walls"):
        c = mesh.boundary_cellsID[f]
        yp = c25 * mesh.face_delta[f] * math.sqrt(k[c]) / 1e-5
        expect = max(1e-5 * (yp * kappa / math.log(max(E * yp, 1.0001)) - 1.0), 0.0) if yp > yl else 0.0
        assert nutf[f] == pytest.approx(expect, rel=1e-13, abs=1e-300)


def sst_channel_case(x, mesh, iterations, precond="Jacobi", transient=False, walls=("walls",)):
    """RANS{KOmegaSST} on a channel (inlet, outlet, walls); omega wall
    functions and k = nut = 0 on the walls; the wall distance's equation
    solved with CG."""
    A = x.api
    model = A.Physics(time=A.Transient() if transient else A.Steady(), fluid=A.Fluid(A.Incompressible, nu=1e-3),
                      turbulence=A.RANS(A.KOmegaSST, walls=list(walls)), energy=A.Energy(A.Isothermal), domain=mesh)
    others = [n for n in mesh.patch_names if n not in ("inlet", "outlet")]
    BCs = A.assign(region=mesh,
                   U=[A.Dirichlet("inlet", [1.0, 0.0, 0.0]), A.Zerogradient("outlet")]
                   + [A.Wall(w, [0.0, 0.0, 0.0]) for w in others],
                   p=[A.Zerogradient("inlet"), A.Dirichlet("outlet", 0.0)] + [A.Wall(w) for w in others],
                   k=[A.Dirichlet("inlet", 0.01), A.Extrapolated("outlet")] + [A.Dirichlet(w, 0.0) for w in others],
                   omega=[A.Dirichlet("inlet", 10.0), A.Extrapolated("outlet")]
                   + [A.OmegaWallFunction(w) for w in others],
                   nut=[A.Dirichlet("inlet", 1e-3), A.Extrapolated("outlet")] + [A.Dirichlet(w, 0.0) for w in others])
    pre = getattr(A, precond)

    def ss(s, relax):
        return A.SolverSetup(solver=s(), preconditioner=pre(), convergence=1e-7, relax=relax, rtol=1e-2)

    tm = A.Euler if transient else A.SteadyState
    config = A.Configuration(
        solvers={"U": ss(A.Bicgstab, 1.0 if transient else 0.7), "p": ss(A.Cg, 1.0 if transient else 0.3),
                 "k": ss(A.Bicgstab, 1.0 if transient else 0.7), "omega": ss(A.Bicgstab, 1.0 if transient else 0.7),
                 "y": A.SolverSetup(solver=A.Cg(), preconditioner=A.Jacobi(), convergence=1e-8, relax=0.9, rtol=1e-3)},
        schemes={"U": A.Schemes(time=tm, divergence=A.Upwind), "p": A.Schemes(),
                 "k": A.Schemes(time=tm, divergence=A.Upwind), "omega": A.Schemes(time=tm, divergence=A.Upwind),
                 "y": A.Schemes()},
        runtime=A.Runtime(iterations=iterations, write_interval=-1, time_step=1e-3 if transient else 1.0),
        hardware=A.Hardware(backend=A.B200Backend()), boundaries=BCs)
    for f, v in ((model.momentum.U, [1.0, 0.0, 0.0]), (model.momentum.p, 0.0), (model.turbulence.k, 0.01),
                 (model.turbulence.omega, 10.0), (model.turbulence.nut, 1e-3)):
        A.initialise_(f, v)
    return model, config


def test_sst_oracle_channel(x, orc):
    """wall_distance! of a square channel is close to the distance to the
    nearest wall by the walls (the Poisson form is exact for a single plane
    wall; on this grid within 15 %) and falls below it towards the centre;
    20 SIMPLE iterations stay finite with positive k, omega and nut;
    coefficient defaults are the reference's."""
    from test_nonorth_oracle import skewed_channel
    A = x.api
    assert A.RANS(A.KOmegaSST, walls=["w"]).coeffs() == dict(beta_star=0.09, alpha1=0.31, sigma_k1=0.85,
                                                              sigma_k2=1.0, sigma_omega1=0.5, sigma_omega2=0.856,
                                                              beta1=0.075, beta2=0.0828, kappa=0.41)
    mesh = skewed_channel(x, n=(16, 10, 8), seed=3, skew=0.0)
    model, config = sst_channel_case(x, mesh, 20)
    cfg, keep = x.build_config(model, config)
    assert cfg.turbulence == x._abi.TURB_KOMEGA_SST and cfg.n_bc_y == 3
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    y = o.get_field(x._abi.FIELD_WALLDIST)
    cc = mesh.cell_centre
    exact = np.minimum.reduce([cc[:, 1], 1 - cc[:, 1], cc[:, 2], 1 - cc[:, 2]])
    near = exact < 0.07
    r = y / exact
    assert np.all(y > 0) and 0.7 < r.min() and r.max() < 1.1
    assert np.max(np.abs(r[near] - 1.0)) < 0.15
    set_komega_fields(x, o, model)
    res, _ = o.simple_iterate(20)
    assert np.all(np.isfinite(res))
    for f in ("FIELD_K", "FIELD_OMEGA", "FIELD_NUT"):
        v = o.get_field(getattr(x._abi, f))
        assert np.all(np.isfinite(v)) and v.min() > 0
