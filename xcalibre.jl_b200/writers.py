"""Result writers: VTK (.vtu) and OpenFOAM case directories.

The formats are the reference's (src/IOFormats/VTK/VTK_writer_3D.jl,
src/IOFormats/OpenFOAM/OpenFOAM_writer.jl):

* VTK: one XML UnstructuredGrid file per write, ASCII, every cell a
  polyhedron (type 42) given by its faces; each face's nodes ordered so its
  normal points out of the cell (the owner's node order, reversed for the
  neighbour).  File ``iteration_<k>.vtu`` for steady runs, ``time_<k>.vtu``
  for transient ones; cell data U (3 components) and p, plus nut for LES.
  A 2D mesh read from a UNV file (a Mesh2 in the reference,
  src/IOFormats/VTK/VTK_writer.jl) is written as a legacy ASCII .vtk file
  (``iteration_<k>.vtk`` / ``time_<k>.vtk``): the points, each cell's nodes
  in element order, cell type 5 (triangle), 9 (quad) or 7 (polygon), and
  SCALARS / VECTORS cell data.
* OpenFOAM: ``constant/polyMesh`` written once, then one time directory per
  write (``<k>`` steady, ``%.8f`` of the time transient) holding
  volVectorField U / volScalarField p with their internal values and one
  boundary entry per patch from the case's boundary conditions (fixedValue
  for Dirichlet / Wall values, empty for Empty, zeroGradient otherwise).

Values are written with 17 significant digits (they read back as the same
doubles).  ``AsyncWriter`` formats and writes files on a background thread,
so the solver keeps running while a write is in progress; the fields it gets
are host copies taken when the write was requested.
"""
from __future__ import annotations

import os
import queue
import threading

import numpy as np

from .meshgen import PolyMesh


def _fmt(a: np.ndarray) -> str:
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1:
        return "\n".join(map(repr, a.tolist())) + "\n"
    return "\n".join(" ".join(map(repr, row)) for row in a.tolist()) + "\n"


class VTKWriter2D:
    """A 2D mesh's .vtk writer: points and the cells' node lists, written
    out in full with the fields at each write (write_results for a Mesh2)."""

    def __init__(self, points, cell_nodes):
        pts = np.asarray(points, dtype=np.float64)
        self.n_cells = len(cell_nodes)
        size = sum(len(c) for c in cell_nodes) + self.n_cells
        types = ["5" if len(c) == 3 else "9" if len(c) == 4 else "7" for c in cell_nodes]
        self.header = (
            "# vtk DataFile Version 3.0\nXCALibre B200 simulation data\nASCII\nDATASET UNSTRUCTURED_GRID\n"
            f"POINTS {pts.shape[0]} double\n" + _fmt(pts)
            + f"CELLS {self.n_cells} {size}\n"
            + "".join(f"{len(c)} " + " ".join(map(str, c)) + "\n" for c in cell_nodes)
            + f"CELL_TYPES {self.n_cells}\n" + "\n".join(types) + "\n"
            + f"CELL_DATA {self.n_cells}\n")

    def write(self, path: str, fields) -> None:
        """fields: [(label, values)] with values [n] (scalar) or [3, n] / [n, 3]."""
        with open(path, "w") as f:
            f.write(self.header)
            for label, v in fields:
                v = np.asarray(v, dtype=np.float64)
                if v.ndim == 2 and v.shape[0] == 3 and v.shape[1] == self.n_cells:
                    v = v.T
                if v.ndim == 1:
                    f.write(f"SCALARS {label} double 1\nLOOKUP_TABLE CellColors\n")
                else:
                    f.write(f"VECTORS {label} double\n")
                f.write(_fmt(v))


class VTKWriter3D:
    """The mesh part of a .vtu file (points and polyhedral cells), built once
    (initialise_writer(VTK(), mesh) in the reference)."""

    def __init__(self, pm: PolyMesh):
        pts = np.asarray(pm.points, dtype=np.float64)
        off = np.asarray(pm.face_offsets, dtype=np.int64)
        nodes = np.asarray(pm.face_nodes, dtype=np.int64)
        owner = np.asarray(pm.owner, dtype=np.int64)
        nei = np.asarray(pm.neighbour, dtype=np.int64)
        nC = pm.n_cells
        # each cell's faces in face order, with "reversed" for the neighbour
        cf = [[] for _ in range(nC)]
        for f in range(owner.size):
            cf[owner[f]].append((f, False))
        for f in range(nei.size):
            cf[nei[f]].append((f, True))
        conn, offsets, faces, faceoffsets = [], [], [], []
        nc = 0
        x = 0
        for c in range(nC):
            seen = {}
            stream = [len(cf[c])]
            for f, rev in cf[c]:
                fn = nodes[off[f]:off[f + 1]].tolist()
                if rev:
                    fn = fn[::-1]
                for v in fn:
                    seen.setdefault(v, None)
                stream.append(len(fn))
                stream.extend(fn)
            conn.append(" ".join(map(str, seen)))
            nc += len(seen)
            offsets.append(nc)
            faces.append(" ".join(map(str, stream)))
            x += len(stream)
            faceoffsets.append(x)
        self.n_cells = nC
        self.header = (
            '<?xml version="1.0"?>\n'
            ' <VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian">\n'
            '  <UnstructuredGrid>\n'
            f'   <Piece NumberOfPoints="{pts.shape[0]}" NumberOfCells="{nC}">\n'
            '    <Points>\n'
            '     <DataArray type="Float64" NumberOfComponents="3" format="ascii">\n'
            + _fmt(pts) +
            '     </DataArray>\n    </Points>\n    <Cells>\n'
            '     <DataArray type="Int64" Name="connectivity" format="ascii">\n' + "\n".join(conn) + "\n"
            '     </DataArray>\n'
            '     <DataArray type="Int64" Name="offsets" format="ascii">\n' + "\n".join(map(str, offsets)) + "\n"
            '     </DataArray>\n'
            '     <DataArray type="Int64" Name="faces" format="ascii">\n' + "\n".join(faces) + "\n"
            '     </DataArray>\n'
            '     <DataArray type="Int64" Name="faceoffsets" format="ascii">\n' + "\n".join(map(str, faceoffsets))
            + "\n     </DataArray>\n"
            '     <DataArray type="UInt8" Name="types" format="ascii">\n' + "42\n" * nC +
            '     </DataArray>\n    </Cells>\n    <CellData>\n')
        self.footer = "    </CellData>\n   </Piece>\n  </UnstructuredGrid>\n </VTKFile>\n"

    def write(self, path: str, fields) -> None:
        """fields: [(label, values)] with values [n] (scalar) or [3, n] / [n, 3]."""
        with open(path, "w") as f:
            f.write(self.header)
            for label, v in fields:
                v = np.asarray(v, dtype=np.float64)
                if v.ndim == 2 and v.shape[0] == 3 and v.shape[1] == self.n_cells:
                    v = v.T
                if v.ndim == 1:
                    f.write(f'     <DataArray type="Float64" Name="{label}" format="ascii">\n')
                else:
                    f.write(f'     <DataArray type="Float64" Name="{label}" format="ascii" '
                            f'NumberOfComponents="{v.shape[1]}">\n')
                f.write(_fmt(v))
                f.write("     </DataArray>\n")
            f.write(self.footer)


def _foam_entry(bc, vector: bool) -> str:
    """_foam_boundary_entry (OpenFOAM_writer.jl:302-360): fixedValue for a
    Dirichlet value and a vector Wall value, empty for Empty, zeroGradient
    for everything else."""
    from . import _abi
    if bc.kind == _abi.BC_EMPTY:
        return "\t{\n\t\ttype empty;\n\t}\n"
    if bc.kind in (_abi.BC_DIRICHLET, _abi.BC_WALL):
        v = np.atleast_1d(np.asarray(bc.value, dtype=np.float64)).tolist()
        if vector and len(v) == 3:
            return f"\t{{\n\t\ttype fixedValue;\n\t\tvalue uniform ({v[0]!r} {v[1]!r} {v[2]!r});\n\t}}\n"
        if not vector and len(v) == 1 and bc.kind == _abi.BC_DIRICHLET:
            return f"\t{{\n\t\ttype fixedValue;\n\t\tvalue uniform {v[0]!r};\n\t}}\n"
    return "\t{\n\t\ttype zeroGradient;\n\t}\n"


class FOAMWriter:
    """An OpenFOAM case directory: constant/polyMesh at construction, one time
    directory per write."""

    def __init__(self, pm: PolyMesh, case_dir: str, bcs: dict):
        from .foamio import write_polymesh
        self.dir = case_dir
        self.n_cells = pm.n_cells
        self.bcs = bcs
        os.makedirs(case_dir, exist_ok=True)
        open(os.path.join(case_dir, "XCALibre.foam"), "a").close()
        write_polymesh(pm, os.path.join(case_dir, "constant", "polyMesh"))

    def write(self, timedir: str, fields) -> None:
        d = os.path.join(self.dir, timedir)
        os.makedirs(d, exist_ok=True)
        for label, v in fields:
            v = np.asarray(v, dtype=np.float64)
            vector = v.ndim == 2
            if vector and v.shape[0] == 3 and v.shape[1] == self.n_cells:
                v = v.T
            cls = "volVectorField" if vector else "volScalarField"
            with open(os.path.join(d, label), "w") as f:
                f.write(f"FoamFile\n{{\n    version     2.0;\n    format      ascii;\n    class       {cls};\n"
                        f"    location    \"{timedir}\";\n    object      {label};\n}}\n")
                f.write(f"internalField   nonuniform List<{'vector' if vector else 'scalar'}>\n"
                        f"{self.n_cells}\n(\n")
                if vector:
                    f.write("\n".join(f"({a!r} {b!r} {c!r})" for a, b, c in v.tolist()) + "\n")
                else:
                    f.write(_fmt(v))
                f.write(");\nboundaryField\n{\n")
                for bc in self.bcs.get(label, []):
                    f.write(f"\t{bc.name}\n" + _foam_entry(bc, vector))
                f.write("}\n")


def _read_foam_internal(path: str) -> np.ndarray:
    """The internalField values of a field file written by FOAMWriter."""
    text = open(path).read()
    a = text.index("internalField")
    b = text.index("(", a)
    e = text.index(");", b)
    body = text[b + 1: e].replace("(", " ").replace(")", " ")
    v = np.array(body.split(), dtype=np.float64)
    return v.reshape(-1, 3) if "List<vector>" in text[a:b] else v


class AsyncWriter:
    """Writes on a background thread: ``submit(fn, *args)`` returns at once;
    ``close()`` waits for every submitted write and re-raises the first
    error."""

    def __init__(self):
        self.q: queue.Queue = queue.Queue()
        self.err = None
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        while True:
            job = self.q.get()
            if job is None:
                return
            fn, args = job
            try:
                fn(*args)
            except Exception as e:  # reported by close()
                if self.err is None:
                    self.err = e

    def submit(self, fn, *args):
        self.q.put((fn, args))

    def close(self):
        self.q.put(None)
        self.t.join()
        if self.err is not None:
            raise self.err
