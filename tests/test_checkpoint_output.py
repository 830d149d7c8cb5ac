"""Checkpoint / restart and result writers on the CPU.

* Restart: a case run N iterations, checkpointed (every readable field, saved
  to an .npz and loaded back), restored into a fresh case that is marked
  initialised, and run N more gives the results of 2N uninterrupted
  iterations bit for bit -- SIMPLE (channel) and PISO (periodic LES), on the
  oracle (the product's restart is checked on the GPU).
* Writers: the .vtu file (the reference's VTK_writer_3D.jl layout: polyhedral
  cells, outward face order) and the OpenFOAM case (polyMesh + time
  directories) read back to the same mesh and field values; meshes read
  from UNV files write too: a 3D one through its polyMesh view (the written
  polyMesh builds the same cells), a 2D one as the legacy .vtk file of
  VTK_writer.jl (points, cell node lists, cell types 5/9/7, cell data)."""
import os
import re
import xml.etree.ElementTree as ET

import numpy as np
import pytest

FIELDS = ("FIELD_U", "FIELD_P", "FIELD_MDOTF", "FIELD_NUEFF", "FIELD_GRADP", "FIELD_GRADU", "FIELD_RD", "FIELD_HV",
          "FIELD_DIVHV", "FIELD_NUT", "FIELD_NUTF", "FIELD_UF", "FIELD_PF", "FIELD_RDF")


def _oracle_case(x, orc, mesh, model, config, pref=None):
    cfg, keep = x.build_config(model, config, pref=pref)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    o.set_field(x._abi.FIELD_U, model.momentum.U)
    o.set_field(x._abi.FIELD_P, model.momentum.p)
    return o, (cfg, keep)


@pytest.mark.parametrize("algo", ["simple", "piso"])
def test_restart_bit_identical_oracle(x, orc, tmp_path, algo):
    if algo == "simple":
        mesh = x.build_mesh3(x.channel_polymesh(10, 6, 5, seed=4, length=2.0))
        mk = lambda: x.cases.channel_case(mesh, iterations=10)
        pref, N = None, 4
    else:
        mesh = x.build_mesh3(x.periodic_box_polymesh(6, seed=2))
        U0 = x.cases.fourier_field(mesh, seed=2)
        mk = lambda: x.cases.periodic_les_case(mesh, steps=6, U0=U0)
        pref, N = 0.0, 3

    def run(c, n):
        return c.simple_iterate(n)[0] if algo == "simple" else c.piso_step(n)[0]

    A = x._abi
    a, ka = _oracle_case(x, orc, mesh, *mk(), pref=pref)
    ra = run(a, 2 * N)
    b, kb = _oracle_case(x, orc, mesh, *mk(), pref=pref)
    rb = run(b, N)
    path = str(tmp_path / "ck.npz")
    x.save_checkpoint({f: b.get_field(getattr(A, f)) for f in FIELDS}, path)
    state = x.load_checkpoint(path)
    c, kc = _oracle_case(x, orc, mesh, *mk(), pref=pref)
    for f in FIELDS:
        c.set_field(getattr(A, f), state[f])
    c.mark_initialised()
    rc = run(c, N)
    assert np.array_equal(np.vstack([rb, rc]), ra)
    for f in ("FIELD_U", "FIELD_P", "FIELD_MDOTF"):
        assert np.array_equal(c.get_field(getattr(A, f)), a.get_field(getattr(A, f))), f
    # without the mark, the restored run redoes the initial calculations (a
    # restart from U and p, as run! does): no longer the same iterates
    d, kd = _oracle_case(x, orc, mesh, *mk(), pref=pref)
    for f in FIELDS:
        d.set_field(getattr(A, f), state[f])
    assert not np.array_equal(run(d, N), rc) or algo == "piso"


def _vtu_arrays(path):
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    arrays = {}
    for da in root.iter("DataArray"):
        name = da.get("Name") or "points"
        arrays[name] = np.array(da.text.split(), dtype=np.float64)
    return int(piece.get("NumberOfCells")), int(piece.get("NumberOfPoints")), arrays


def test_vtu_writer(x, tmp_path):
    from importlib import import_module
    W = import_module(x.__name__ + ".writers")
    pm = x.box_polymesh(4, 3, 2, seed=5)
    mesh = x.build_mesh3(pm)
    w = W.VTKWriter3D(pm)
    rng = np.random.default_rng(0)
    U = rng.standard_normal((3, mesh.n_cells))
    p = rng.standard_normal(mesh.n_cells)
    path = str(tmp_path / "iteration_3.vtu")
    w.write(path, [("U", U), ("p", p)])
    nc, npt, arr = _vtu_arrays(path)
    assert nc == mesh.n_cells and npt == len(pm.points)
    assert np.array_equal(arr["points"].reshape(-1, 3), np.asarray(pm.points))
    assert np.array_equal(arr["U"].reshape(-1, 3), U.T) and np.array_equal(arr["p"], p)
    assert np.all(arr["types"] == 42)
    # every cell's faces are outward: the node-order normal points away from
    # the cell centre
    faces, fo = arr["faces"].astype(int), arr["faceoffsets"].astype(int)
    pts = np.asarray(pm.points)
    start = 0
    for c in range(nc):
        s = faces[start: fo[c]]
        k, pos = s[0], 1
        assert k == 6
        for _ in range(k):
            m = s[pos]
            q = pts[s[pos + 1: pos + 1 + m]]
            nrm = np.cross(q[1] - q[0], q[2] - q[0])
            assert np.dot(nrm, q.mean(axis=0) - mesh.cell_centre[c]) > 0
            pos += 1 + m
        start = fo[c]


def test_foam_writer(x, tmp_path):
    from importlib import import_module
    W = import_module(x.__name__ + ".writers")
    pm = x.cavity_polymesh(5, seed=1)
    mesh = x.build_mesh3(pm)
    model, config = x.cases.cavity_case(mesh, iterations=1)
    w = W.FOAMWriter(pm, str(tmp_path), config.boundaries)
    rng = np.random.default_rng(1)
    U = rng.standard_normal((3, mesh.n_cells))
    p = rng.standard_normal(mesh.n_cells)
    w.write("7", [("U", U), ("p", p)])
    back = x.read_polymesh(str(tmp_path / "constant" / "polyMesh"))
    assert np.array_equal(back.points, pm.points) and np.array_equal(back.owner, pm.owner)
    assert np.array_equal(W._read_foam_internal(str(tmp_path / "7" / "U")), U.T)
    assert np.array_equal(W._read_foam_internal(str(tmp_path / "7" / "p")), p)
    txt = open(tmp_path / "7" / "U").read()
    assert re.search(r"lid\s*\{\s*type fixedValue;\s*value uniform \(1\.0 0\.0 0\.0\);", txt)
    assert re.search(r"frontAndBack\s*\{\s*type empty;", txt)
    assert os.path.exists(tmp_path / "XCALibre.foam")


def test_unv3_mesh_writers(x, tmp_path):
    """A 3D UNV mesh (the hex cavity) writes its .vtu (outward faces) and its
    OpenFOAM case; the written polyMesh builds a mesh with the same cell
    volumes and centres."""
    from importlib import import_module
    from test_unv3 import unv3_fixture_mesh
    W = import_module(x.__name__ + ".writers")
    m = unv3_fixture_mesh(x, "cavity_hex_unv3.npz")
    pm = m.polymesh
    assert pm is not None and pm.n_cells == m.n_cells and pm.n_faces == m.n_faces
    assert np.all(pm.owner[:pm.n_internal_faces] < pm.neighbour)
    w = W.VTKWriter3D(pm)
    rng = np.random.default_rng(3)
    U = rng.standard_normal((3, m.n_cells))
    p = rng.standard_normal(m.n_cells)
    path = str(tmp_path / "iteration_1.vtu")
    w.write(path, [("U", U), ("p", p)])
    nc, npt, arr = _vtu_arrays(path)
    assert nc == m.n_cells and np.array_equal(arr["p"], p)
    faces, fo = arr["faces"].astype(int), arr["faceoffsets"].astype(int)
    pts = np.asarray(pm.points)
    start = 0
    for c in range(nc):
        s = faces[start: fo[c]]
        k, pos = s[0], 1
        for _ in range(k):
            n_ = s[pos]
            q = pts[s[pos + 1: pos + 1 + n_]]
            nrm = np.cross(q[1] - q[0], q[2] - q[0])
            assert np.dot(nrm, q.mean(axis=0) - m.cell_centre[c]) > 0
            pos += 1 + n_
        start = fo[c]
    bcs = {name: [] for name in m.patch_names}
    fw = W.FOAMWriter(pm, str(tmp_path / "foam"), bcs)
    fw.write("1", [("U", U), ("p", p)])
    back = x.build_mesh3(x.read_polymesh(str(tmp_path / "foam" / "constant" / "polyMesh")))
    assert back.n_cells == m.n_cells
    assert np.allclose(back.cell_volume, m.cell_volume, rtol=1e-12, atol=0)
    assert np.allclose(back.cell_centre, m.cell_centre, rtol=0, atol=1e-12)


def test_unv2_vtk_writer(x, tmp_path):
    """A 2D UNV mesh (the 10 mm backward-facing step) writes the legacy .vtk
    of VTK_writer.jl: POINTS, CELLS with each cell's nodes, CELL_TYPES,
    SCALARS / VECTORS cell data."""
    from importlib import import_module
    from test_unv import bfs_mesh
    W = import_module(x.__name__ + ".writers")
    m = bfs_mesh(x, 10)
    assert m.dim == 2 and m.polymesh is None and len(m.cell_nodes) == m.n_cells
    w = W.VTKWriter2D(m.points, m.cell_nodes)
    rng = np.random.default_rng(4)
    U = rng.standard_normal((3, m.n_cells))
    p = rng.standard_normal(m.n_cells)
    path = str(tmp_path / "iteration_2.vtk")
    w.write(path, [("U", U), ("p", p)])
    lines = open(path).read().split("\n")
    assert lines[0] == "# vtk DataFile Version 3.0" and lines[2] == "ASCII"
    assert lines[3] == "DATASET UNSTRUCTURED_GRID"
    npt = len(m.points)
    assert lines[4] == f"POINTS {npt} double"
    assert np.array_equal(np.array([l.split() for l in lines[5:5 + npt]], dtype=np.float64), m.points)
    k = 5 + npt
    size = sum(len(c) for c in m.cell_nodes) + m.n_cells
    assert lines[k] == f"CELLS {m.n_cells} {size}"
    for c in range(m.n_cells):
        row = list(map(int, lines[k + 1 + c].split()))
        assert row[0] == len(m.cell_nodes[c]) and row[1:] == list(m.cell_nodes[c])
    k += 1 + m.n_cells
    assert lines[k] == f"CELL_TYPES {m.n_cells}"
    types = list(map(int, lines[k + 1: k + 1 + m.n_cells]))
    assert all(t == {3: 5, 4: 9}.get(len(cn), 7) for t, cn in zip(types, m.cell_nodes))
    k += 1 + m.n_cells
    assert lines[k] == f"CELL_DATA {m.n_cells}"
    assert lines[k + 1] == "VECTORS U double"
    got_U = np.array([l.split() for l in lines[k + 2: k + 2 + m.n_cells]], dtype=np.float64)
    assert np.array_equal(got_U, U.T)
    k += 2 + m.n_cells
    assert lines[k] == "SCALARS p double 1" and lines[k + 1] == "LOOKUP_TABLE CellColors"
    assert np.array_equal(np.array(lines[k + 2: k + 2 + m.n_cells], dtype=np.float64), p)
