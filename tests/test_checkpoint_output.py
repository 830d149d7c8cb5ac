"""Checkpoint / restart and result writers on the CPU.

* Restart: a case run N iterations, checkpointed (every readable field, saved
  to an .npz and loaded back), restored into a fresh case that is marked
  initialised, and run N more gives the results of 2N uninterrupted
  iterations bit for bit -- SIMPLE (channel) and PISO (periodic LES), on the
  oracle (the product's restart is checked on the GPU).
* Writers: the .vtu file (the reference's VTK_writer_3D.jl layout: polyhedral
  cells, outward face order) and the OpenFOAM case (polyMesh + time
  directories) read back to the same mesh and field values."""
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
