"""2D UNV meshes (UNV2D_mesh, src/UNV2) and the Jacobi smoother on the CPU.

* the reference's own grids, read in place where its checkout is present:
  the counts test/test_mesh_conversion.jl:27-41 expects (trig40 3484 cells /
  5306 faces / 1823 nodes, quad40 1600 / 3280 / 1681), closed cells and the
  domain area; laplace_unit_3by3.unv assembled into the exact A and b of
  test/unit_test_laplace.jl:112-130, in the reference's own cell order;
* the backward-facing-step grid of
  test/0_TEST_CASES/2d_incompressible_laminar_BFS.jl from its committed raw
  parse: 500 SIMPLE iterations (Jacobi smoother, 5 sweeps, omega 2/3) on the
  oracle meet the test's known answer, outlet Ux = 0.5 inlet Ux +- 0.05;
* the smoother's 5x5 system of test/test_smoothers.jl:31-46: 50 sweeps with
  omega 1 from zero reach A\\b to 0.1; its constructors (:1-28)."""
import json
import os

import numpy as np
import pytest

from refpath import ref_path
from test_oracle_golden import GOLD

GRIDS = ref_path("test", "grids")
EX = ref_path("examples", "0_GRIDS")


def bfs_mesh(x, mm=10):
    """backwardFacingStep_<mm>mm.unv (scale 0.001) from tests/golden/bfs_<mm>mm_unv.npz."""
    d = np.load(os.path.join(GOLD, "bfs_%dmm_unv.npz" % mm))
    verts = d["elem_vertices"] - 1
    off = np.concatenate([[0], np.cumsum(d["elem_count"])])
    elements = [(int(i), int(c), verts[off[k]:off[k + 1]].tolist())
                for k, (i, c) in enumerate(zip(d["elem_index"], d["elem_count"]))]
    go = d["group_offsets"]
    groups = [(str(n), d["group_elements"][go[k]:go[k + 1]].tolist()) for k, n in enumerate(d["group_names"])]
    return x.unv.unv2_mesh(d["points"], elements, groups, scale=0.001)


def bfs_case(x, mesh, iterations=500, smoother=True):
    """2d_incompressible_laminar_BFS.jl:11-80: Umag 0.5, nu 1e-3, Linear
    divergence for U, BiCGSTAB/CG with Jacobi, relax 0.8/0.2, rtol 0.1/0.01."""
    A = x.api
    Umag = 0.5
    model = A.Physics(time=A.Steady(), fluid=A.Fluid(A.Incompressible, nu=1e-3), turbulence=A.RANS(A.Laminar),
                      energy=A.Energy(A.Isothermal), domain=mesh)
    BCs = A.assign(region=mesh,
                   U=[A.Dirichlet("inlet", [Umag, 0.0, 0.0]), A.Extrapolated("outlet"), A.Wall("wall", [0.0, 0.0, 0.0]),
                      A.Symmetry("top")],
                   p=[A.Extrapolated("inlet"), A.Dirichlet("outlet", 0.0), A.Extrapolated("wall"), A.Symmetry("top")])

    def sm():
        return A.JacobiSmoother(domain=mesh, loops=5, omega=2 / 3) if smoother else None

    solvers = {"U": A.SolverSetup(solver=A.Bicgstab(), smoother=sm(), preconditioner=A.Jacobi(), convergence=1e-7,
                                  relax=0.8, rtol=1e-1),
               "p": A.SolverSetup(solver=A.Cg(), smoother=sm(), preconditioner=A.Jacobi(), convergence=1e-7,
                                  relax=0.2, rtol=1e-2)}
    config = A.Configuration(solvers=solvers, schemes={"U": A.Schemes(divergence=A.Linear), "p": A.Schemes()},
                             runtime=A.Runtime(iterations=iterations, time_step=1, write_interval=iterations),
                             hardware=A.Hardware(backend=A.B200Backend()), boundaries=BCs)
    A.initialise_(model.momentum.U, [Umag, 0.0, 0.0])
    A.initialise_(model.momentum.p, 0.0)
    return model, config


def check_bfs_answer(x, U, config, mesh):
    inlet = x.api.boundary_average("inlet", U, config.boundaries["U"], mesh=mesh)
    outlet = x.api.boundary_average("outlet", U, config.boundaries["U"], mesh=mesh)
    assert inlet[0] == pytest.approx(0.5)
    # isapprox(outlet, 0.5 inlet; atol = 0.1 Umag): the norm of the difference
    assert np.linalg.norm(outlet - 0.5 * inlet) <= 0.05, (inlet, outlet)


def _closure(m):
    S = m.face_normal * m.face_area[:, None]
    acc = np.zeros((m.n_cells, 3))
    cells = np.repeat(np.arange(m.n_cells), np.diff(m.cell_faces_offset))
    np.add.at(acc, cells, S[m.cell_faces] * m.cell_nsign[:, None])
    np.add.at(acc, m.boundary_cellsID, S[:m.n_bfaces])
    return np.abs(acc).max() / np.abs(S).max()


@pytest.mark.skipif(not os.path.isdir(GRIDS), reason="XCAL_REFERENCE_DIR (an XCALibre.jl checkout) not set")
@pytest.mark.parametrize("grid,counts", [("trig40.unv", (3484, 5306, 1823)), ("quad40.unv", (1600, 3280, 1681))])
def test_reference_grid_counts(x, grid, counts):
    m = x.UNV2D_mesh(os.path.join(GRIDS, grid), scale=0.001)
    assert str(m) == "2D Mesh with:\n-> %d cells\n-> %d faces\n-> %d nodes" % counts
    assert m.dim == 2 and m.patch_names == ["inlet", "outlet", "bottom", "top"]
    assert _closure(m) < 1e-12
    assert abs(m.cell_volume.sum() - 1.0) < 1e-12 and m.cell_volume.min() > 0
    assert np.all(np.abs(m.face_normal[:, 2]) == 0.0) and np.all(m.face_weight[: m.n_bfaces] == 1.0)


@pytest.mark.skipif(not os.path.isdir(EX), reason="XCAL_REFERENCE_DIR (an XCALibre.jl checkout) not set")
def test_laplace_unit_3by3_unv(x, orc):
    """unit_test_laplace.jl on its own mesh: -Laplacian(k=1, T) == 0 as the p
    equation (rDf = 1), A and b compared in the reference's cell order."""
    m = x.UNV2D_mesh(os.path.join(EX, "laplace_unit_3by3.unv"))
    assert (m.n_cells, m.n_faces) == (9, 24)
    A_ = x.api
    model = A_.Physics(time=A_.Steady(), fluid=A_.Fluid(A_.Incompressible, nu=1.0), turbulence=A_.RANS(A_.Laminar),
                       energy=A_.Energy(A_.Isothermal), domain=m)
    BCs = A_.assign(region=m, U=[A_.Zerogradient(n) for n in m.patch_names],
                    p=[A_.Dirichlet("left_wall", 50.0), A_.Zerogradient("upper_wall"), A_.Zerogradient("right_wall"),
                       A_.Dirichlet("bottom_wall", 10.0)])
    solvers = {"U": A_.SolverSetup(solver=A_.Bicgstab(), preconditioner=A_.Jacobi(), convergence=1e-8, relax=0.8),
               "p": A_.SolverSetup(solver=A_.Cg(), preconditioner=A_.Jacobi(), convergence=1e-8, relax=0.8)}
    config = A_.Configuration(solvers=solvers, schemes={"U": A_.Schemes(), "p": A_.Schemes()},
                              runtime=A_.Runtime(iterations=1, write_interval=1, time_step=1.0),
                              hardware=A_.Hardware(backend=A_.B200Backend()), boundaries=BCs)
    cfg, keep = x.build_config(model, config)
    oc = orc.OracleCase(orc.OracleMesh.from_mesh3(m), cfg)
    oc.discretise(1)
    oc.apply_boundary_conditions(1)
    rp, cv = oc.pattern(1)
    nz, b = oc.system(1)
    Am = np.zeros((9, 9))
    for i in range(9):
        Am[i, cv[rp[i]:rp[i + 1]]] = nz[rp[i]:rp[i + 1]]
    g = json.load(open(os.path.join(GOLD, "laplace_3by3.json")))
    assert np.allclose(Am, np.array(g["A"]), atol=g["atol_A"], rtol=0)
    assert np.allclose(b, np.array(g["b"]), rtol=1.5e-8, atol=0)


@pytest.mark.skipif(not os.path.isdir(EX), reason="XCAL_REFERENCE_DIR (an XCALibre.jl checkout) not set")
def test_bfs_fixture_matches_file(x):
    a = x.UNV2D_mesh(os.path.join(EX, "backwardFacingStep_10mm.unv"), scale=0.001)
    b = bfs_mesh(x)
    for k in ("face_owner", "face_neigh", "face_centre", "face_normal", "face_e", "face_area", "face_delta",
              "face_weight", "cell_centre", "cell_volume", "cell_faces_offset", "cell_faces", "cell_nsign",
              "cell_neighbours", "boundary_cellsID", "patch_start", "patch_count"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_bfs_laminar_known_answer(x, orc):
    mesh = bfs_mesh(x)
    assert (mesh.n_cells, mesh.patch_names) == (1800, ["inlet", "outlet", "wall", "top"])
    assert _closure(mesh) < 1e-12
    model, config = bfs_case(x, mesh)
    cfg, keep = x.build_config(model, config)
    assert cfg.U_solver.smoother_loops == 5 and cfg.p_solver.smoother_omega == 2 / 3
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    o.set_field(x._abi.FIELD_U, model.momentum.U)
    o.set_field(x._abi.FIELD_P, model.momentum.p)
    res, _ = o.simple_iterate(500)
    assert np.all(np.isfinite(res)) and np.all(res[:, 2] == 0.0)  # z: zero right-hand side on a 2D mesh
    U = o.get_field(x._abi.FIELD_U)
    assert np.all(U[2] == 0.0)
    check_bfs_answer(x, U, config, mesh)


def test_smoother_golden(orc):
    g = json.load(open(os.path.join(GOLD, "smoother_5x5.json")))
    A = np.zeros((5, 5))
    for i, j, v in zip(g["i"], g["j"], g["v"]):
        A[i - 1, j - 1] += v
    rp, cv, nz = [0], [], []
    for r in range(5):
        cols = np.nonzero(A[r])[0]
        cv += cols.tolist()
        nz += A[r, cols].tolist()
        rp.append(len(cv))
    b = np.array(g["b"])
    xs = orc.jacobi_smooth(rp, cv, nz, b, np.zeros(5), g["loops"], g["omega"])
    assert np.allclose(xs, np.linalg.solve(A, b), atol=g["atol"], rtol=0)
    # one sweep by hand: x1_i = omega/a_ii (b_i - sum_{j!=i} a_ij x0_j) + (1 - omega) x0_i
    x0 = np.linspace(1.0, 2.0, 5)
    x1 = orc.jacobi_smooth(rp, cv, nz, b, x0, 1, 2 / 3)
    d = np.diag(A)
    assert np.allclose(x1, (2 / 3) / d * (b - (A @ x0 - d * x0)) + (1 / 3) * x0, rtol=1e-14)


def test_smoother_constructors(x):
    m = x.build_mesh3(x.cavity_polymesh(4))
    s = x.JacobiSmoother(m)
    assert (s.loops, s.omega) == (5, 1.0)
    s = x.JacobiSmoother(domain=m, loops=5)
    assert s.loops == 5 and s.omega == pytest.approx(2 / 3)
    s = x.JacobiSmoother(5, 1, np.zeros(10))
    assert (s.loops, s.omega) == (5, 1.0)
    with pytest.raises(TypeError):
        x.JacobiSmoother(loops=3)
