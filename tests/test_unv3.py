"""3D UNV meshes (UNV3D_mesh, src/UNV3) on the CPU.

* test/test_mesh_conversion.jl:43-61: cavity_hex.unv gives "3D Mesh with:
  125 cells, 450 faces, 216 nodes", the same string as the cavity's
  polyMesh (both read in place where the reference checkout is present);
* the committed raw parses (hex cavity, tetrahedral streamtube) build the
  same mesh as the files; cells close (sum of n S = 0 up to the reference's
  1e-16 regularisation of the face normal) and fill their bounding box;
* SIMPLE runs on the cavity and the tetrahedra (oracle)."""
import os

import numpy as np
import pytest

from refpath import ref_path
from test_oracle_golden import GOLD

CAV_UNV = ref_path("test/grids/OF_cavity_hex/cavity_hex.unv")
CAV_FOAM = ref_path("test/grids/OF_cavity_hex/polyMesh")
TUBE = ref_path("examples/0_GRIDS/3d_streamtube_1.0x0.1x0.1_0.08mm.unv")


def unv3_fixture_mesh(x, name, scale=0.001):
    d = np.load(os.path.join(GOLD, name))

    def split(counts, verts):
        off = np.concatenate([[0], np.cumsum(counts)])
        return [(verts[off[k]:off[k + 1]] - 1).tolist() for k in range(len(counts))]

    faces = split(d["face_count"], d["face_vertices"])
    cells = split(d["cell_count"], d["cell_vertices"])
    go = d["group_offsets"]
    groups = [(str(n), d["group_faces"][go[k]:go[k + 1]].tolist()) for k, n in enumerate(d["group_names"])]
    return x.unv.unv3_mesh(d["points"] * scale, faces, cells, groups)


def _closure(m):
    S = m.face_normal * m.face_area[:, None]
    acc = np.zeros((m.n_cells, 3))
    cells = np.repeat(np.arange(m.n_cells), np.diff(m.cell_faces_offset))
    np.add.at(acc, cells, S[m.cell_faces] * m.cell_nsign[:, None])
    np.add.at(acc, m.boundary_cellsID, S[:m.n_bfaces])
    return np.abs(acc).max() / np.abs(S).max()


ARRAYS = ("face_owner", "face_neigh", "face_centre", "face_normal", "face_e", "face_area", "face_delta",
          "face_weight", "cell_centre", "cell_volume", "cell_faces_offset", "cell_faces", "cell_nsign",
          "cell_neighbours", "boundary_cellsID", "patch_start", "patch_count")


@pytest.mark.skipif(not os.path.isfile(CAV_UNV), reason="XCAL_REFERENCE_DIR (an XCALibre.jl checkout) not set")
def test_cavity_hex_unv_matches_foam_counts(x):
    u = x.UNV3D_mesh(CAV_UNV, scale=0.001)
    f = x.FOAM3D_mesh(CAV_FOAM, scale=0.001)
    assert str(u) == str(f) == "3D Mesh with:\n-> 125 cells\n-> 450 faces\n-> 216 nodes"
    b = unv3_fixture_mesh(x, "cavity_hex_unv3.npz")
    for k in ARRAYS:
        assert np.array_equal(getattr(u, k), getattr(b, k)), k


@pytest.mark.skipif(not os.path.isfile(TUBE), reason="XCAL_REFERENCE_DIR (an XCALibre.jl checkout) not set")
def test_streamtube_fixture_matches_file(x):
    u = x.UNV3D_mesh(TUBE, scale=0.001)
    b = unv3_fixture_mesh(x, "streamtube_unv3.npz")
    assert (u.n_cells, u.n_faces) == (618, 1485)
    for k in ARRAYS:
        assert np.array_equal(getattr(u, k), getattr(b, k)), k


@pytest.mark.parametrize("name,tol", [("cavity_hex_unv3.npz", 1e-14), ("streamtube_unv3.npz", 1e-7)])
def test_unv3_geometry(x, name, tol):
    m = unv3_fixture_mesh(x, name, scale=1.0)
    assert m.dim == 3 and _closure(m) < tol
    ext = np.ptp(m.points, axis=0)
    assert abs(m.cell_volume.sum() / np.prod(ext) - 1.0) < tol
    assert m.cell_volume.min() > 0
    # internal faces point from owner to neighbour, boundary faces out of the owner
    cc, fc, n = m.cell_centre, m.face_centre, m.face_normal
    i = np.arange(m.n_bfaces, m.n_faces)
    assert np.all(np.sum((cc[m.face_neigh[i]] - cc[m.face_owner[i]]) * n[i], axis=1) > 0)


@pytest.mark.parametrize("name", ["cavity_hex_unv3.npz", "streamtube_unv3.npz"])
def test_unv3_simple_oracle(x, orc, name):
    mesh = unv3_fixture_mesh(x, name)
    model, config = unv3_case(x, mesh, 15)
    cfg, keep = x.build_config(model, config, pref=0.0 if name.startswith("cavity") else None)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    o.set_field(x._abi.FIELD_U, model.momentum.U)
    o.set_field(x._abi.FIELD_P, model.momentum.p)
    res, _ = o.simple_iterate(15)
    assert np.all(np.isfinite(res)) and res[-1, 0] < res[0, 0]


def unv3_case(x, mesh, iterations):
    """Lid-driven cube on the cavity ("top" moving), or a through-flow on the
    streamtube (inlet -> outlet, walls elsewhere)."""
    A = x.api
    model = A.Physics(time=A.Steady(), fluid=A.Fluid(A.Incompressible, nu=1e-3), turbulence=A.RANS(A.Laminar),
                      energy=A.Energy(A.Isothermal), domain=mesh)
    if "top" in mesh.patch_names and len(mesh.patch_names) == 2:
        BCs = A.assign(region=mesh, U=[A.Wall("walls", [0.0, 0.0, 0.0]), A.Wall("top", [1e-3, 0.0, 0.0])],
                       p=[A.Wall("walls"), A.Wall("top")])
    else:
        walls = [n for n in mesh.patch_names if n not in ("inlet", "outlet")]
        BCs = A.assign(region=mesh, U=[A.Dirichlet("inlet", [1e-3, 0.0, 0.0]), A.Zerogradient("outlet")]
                       + [A.Wall(w, [0.0, 0.0, 0.0]) for w in walls],
                       p=[A.Zerogradient("inlet"), A.Dirichlet("outlet", 0.0)] + [A.Wall(w) for w in walls])
    solvers = {"U": A.SolverSetup(solver=A.Bicgstab(), preconditioner=A.DILU(), convergence=1e-7, relax=0.7),
               "p": A.SolverSetup(solver=A.Cg(), preconditioner=A.Jacobi(), convergence=1e-7, relax=0.3)}
    config = A.Configuration(solvers=solvers, schemes={"U": A.Schemes(divergence=A.Upwind), "p": A.Schemes()},
                             runtime=A.Runtime(iterations=iterations, write_interval=-1, time_step=1.0),
                             hardware=A.Hardware(backend=A.B200Backend()), boundaries=BCs)
    return model, config
