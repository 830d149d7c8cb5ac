"""OpenFOAM polyMesh files: write -> read round trips of the generated meshes
give the same PolyMesh and the same Mesh3; the reference's own test grid
(test/grids/OF_cavity_hex/polyMesh, read in place where the reference
checkout is present) gives the counts its mesh-conversion test expects
(test/test_mesh_conversion.jl:51-57: 125 cells, 450 faces, 216 nodes), and
the SIMPLE path runs on it (CPU oracle)."""
import os

import numpy as np
import pytest
from refpath import ref_path

REF_CAVITY = ref_path("test/grids/OF_cavity_hex/polyMesh")

MESH3_FIELDS = ["face_owner", "face_neigh", "face_centre", "face_normal", "face_e", "face_area", "face_delta",
                "face_weight", "cell_centre", "cell_volume", "cell_faces_offset", "cell_faces", "cell_nsign",
                "cell_neighbours", "boundary_cellsID", "patch_start", "patch_count"]


@pytest.mark.parametrize("kind", ["cavity", "channel", "periodic"])
def test_polymesh_round_trip(x, tmp_path, kind):
    if kind == "cavity":
        pm = x.cavity_polymesh(9, seed=3, nx=12, lx=1.3)
    elif kind == "channel":
        pm = x.channel_polymesh(10, 6, 5, seed=4, length=2.0)
    else:
        pm = x.periodic_box_polymesh(6, seed=2)
    d = str(tmp_path / "polyMesh")
    x.write_polymesh(pm, d)
    back = x.read_polymesh(d)
    for k in ("points", "face_offsets", "face_nodes", "owner", "neighbour"):
        assert np.array_equal(getattr(pm, k), getattr(back, k)), k
    assert back.patch_names == list(pm.patch_names) and back.patch_sizes == list(pm.patch_sizes)
    a, b = x.build_mesh3(pm), x.FOAM3D_mesh(d)
    assert (a.n_cells, a.n_faces, a.n_bfaces) == (b.n_cells, b.n_faces, b.n_bfaces)
    for k in MESH3_FIELDS:
        if hasattr(a, k):
            assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_scale_and_errors(x, tmp_path):
    pm = x.cavity_polymesh(4)
    d = str(tmp_path / "pm")
    x.write_polymesh(pm, d)
    assert np.array_equal(x.read_polymesh(d, scale=0.001).points, 0.001 * np.asarray(pm.points))
    # a patch that does not start where the previous one ends is refused
    bfile = os.path.join(d, "boundary")
    txt = open(bfile).read()
    start = int(np.asarray(pm.neighbour).size)
    open(bfile, "w").write(txt.replace(f"startFace       {start};", f"startFace       {start + 1};", 1))
    with pytest.raises(ValueError):
        x.read_polymesh(d)


@pytest.mark.skipif(not os.path.isdir(REF_CAVITY), reason="XCAL_REFERENCE_DIR (an XCALibre.jl checkout) not set")
def test_reference_cavity_grid(x, orc):
    pm = x.read_polymesh(REF_CAVITY, scale=0.001)
    mesh = x.FOAM3D_mesh(REF_CAVITY, scale=0.001)
    assert (mesh.n_cells, mesh.n_faces, pm.points.shape[0]) == (125, 450, 216)
    assert pm.patch_names == ["walls", "top"] and pm.patch_sizes == [125, 25]
    # a cube (the points' bounding box) filled exactly by the cells
    ext = np.ptp(np.asarray(pm.points), axis=0)
    assert abs(mesh.cell_volume.sum() / np.prod(ext) - 1.0) < 1e-12
    assert str(mesh) == "3D Mesh with:\n-> 125 cells\n-> 450 faces\n-> 216 nodes"
    # the SIMPLE path on it: lid-driven cube (lid = "top"), CPU oracle
    A = x.api
    model = A.Physics(time=A.Steady(), fluid=A.Fluid(A.Incompressible, nu=0.001), turbulence=A.RANS(A.Laminar),
                      energy=A.Energy(A.Isothermal), domain=mesh)
    BCs = A.assign(region=mesh, U=[A.Wall("walls", [0.0, 0.0, 0.0]), A.Wall("top", [1.0, 0.0, 0.0])],
                   p=[A.Wall("walls"), A.Wall("top")])
    solvers = {"U": A.SolverSetup(solver=A.Bicgstab(), preconditioner=A.DILU(), convergence=1e-7, relax=0.7),
               "p": A.SolverSetup(solver=A.Cg(), preconditioner=A.Jacobi(), convergence=1e-7, relax=0.3)}
    config = A.Configuration(solvers=solvers, schemes={"U": A.Schemes(divergence=A.Upwind), "p": A.Schemes()},
                             runtime=A.Runtime(iterations=30, write_interval=-1, time_step=1.0),
                             hardware=A.Hardware(backend=A.B200Backend()), boundaries=BCs)
    A.initialise_(model.momentum.U, [0.0, 0.0, 0.0])
    A.initialise_(model.momentum.p, 0.0)
    cfg, keep = x.build_config(model, config, pref=0.0)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    o.set_field(x._abi.FIELD_U, model.momentum.U)
    o.set_field(x._abi.FIELD_P, model.momentum.p)
    res, _ = o.simple_iterate(30)
    assert res.shape == (30, 4) and np.all(np.isfinite(res))
    assert res[-1, 0] < res[0, 0] and res[-1, 3] < res[0, 3]
