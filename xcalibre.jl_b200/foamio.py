"""OpenFOAM polyMesh files (ASCII) <-> PolyMesh, and ``FOAM3D_mesh``.

``read_polymesh`` reads a ``constant/polyMesh`` directory the way
``read_FOAM3D`` does (src/FoamMesh/FoamMesh_1_read.jl:1-222):

* every file's data starts after its first line that holds nothing but an
  integer (the entry count), which skips the FoamFile header;
* ``points``: one ``(x y z)`` per entry, each coordinate multiplied by
  ``scale`` (``scale * parse(value)``, :204-217);
* ``faces``: ``n(v0 v1 ...)`` per face (:110-140);
* ``owner`` / ``neighbour``: one cell index per face / internal face
  (:142-176); boundary faces are the faces past the neighbour list (:27-42);
* ``boundary``: per patch its name, ``nFaces`` and ``startFace`` (:44-87).

Indices stay 0-based here (the reference shifts to 1-based).  Patches must be
contiguous and follow the internal faces, which is how OpenFOAM writes them
and what the mesh builder (FoamMesh_2_connect.jl .. FoamMesh_5_build.jl)
assumes.  Binary-format files are refused with an error.

``write_polymesh`` writes the same five files (ASCII), so a generated mesh
can be stored and read back, or handed to OpenFOAM tools.
"""
from __future__ import annotations

import os
import re

import numpy as np

from .foam import Mesh3, build_mesh3
from .meshgen import PolyMesh

_INT_LINE = re.compile(r"^\s*(\d+)\s*$")


def _data_after_count(path: str) -> tuple[int, str]:
    """(entry count, the text after the count line) of one polyMesh file."""
    with open(path, "r") as f:
        text = f.read()
    head = text[: text.find("\n(") + 1] if "\n(" in text else text
    if re.search(r"\bformat\s+binary\s*;", head):
        raise ValueError(f"{path}: binary polyMesh files are not supported (write it as ascii)")
    pos = 0
    for line in text.splitlines(keepends=True):
        m = _INT_LINE.match(line)
        pos += len(line)
        if m:
            return int(m.group(1)), text[pos:]
    raise ValueError(f"{path}: no entry count line")


def _body(rest: str) -> str:
    """The list between the opening '(' and its matching ')'."""
    a = rest.find("(")
    if a < 0:
        raise ValueError("polyMesh list: missing '('")
    depth = 0
    for k in range(a, len(rest)):
        c = rest[k]
        if c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
            if depth == 0:
                return rest[a + 1: k]
    raise ValueError("polyMesh list: unbalanced parentheses")


def _ints(s: str) -> np.ndarray:
    s = s.replace("(", " ").replace(")", " ")
    return np.array(s.split(), dtype=np.int64)


def _read_points(path: str, scale: float) -> np.ndarray:
    n, rest = _data_after_count(path)
    vals = np.array(_body(rest).replace("(", " ").replace(")", " ").split(), dtype=np.float64)
    if vals.size != 3 * n:
        raise ValueError(f"{path}: expected {n} points, found {vals.size / 3:g}")
    return (scale * vals).reshape(n, 3)


def _read_faces(path: str) -> tuple[np.ndarray, np.ndarray]:
    n, rest = _data_after_count(path)
    t = _ints(_body(rest))
    # fast path: every face has the same node count m
    if t.size and t.size % (int(t[0]) + 1) == 0 and t.size // (int(t[0]) + 1) == n:
        m = int(t[0])
        tt = t.reshape(n, m + 1)
        if np.all(tt[:, 0] == m):
            offsets = np.arange(n + 1, dtype=np.int64) * m
            return offsets.astype(np.int32), tt[:, 1:].reshape(-1).astype(np.int32)
    offsets = np.zeros(n + 1, dtype=np.int64)
    nodes = []
    p = 0
    for f in range(n):
        k = int(t[p])
        nodes.append(t[p + 1: p + 1 + k])
        offsets[f + 1] = offsets[f] + k
        p += 1 + k
    if p != t.size:
        raise ValueError(f"{path}: face list does not match its count {n}")
    return offsets.astype(np.int32), np.concatenate(nodes).astype(np.int32)


def _read_labels(path: str) -> np.ndarray:
    n, rest = _data_after_count(path)
    v = _ints(_body(rest))
    if v.size != n:
        raise ValueError(f"{path}: expected {n} labels, found {v.size}")
    return v.astype(np.int32)


def _read_boundary(path: str) -> list[tuple[str, int, int]]:
    n, rest = _data_after_count(path)
    body = _body(rest)
    patches = []
    for m in re.finditer(r"([A-Za-z_][\w.:\-]*)\s*\{([^{}]*)\}", body):
        name, block = m.group(1), m.group(2)
        nf = re.search(r"\bnFaces\s+(\d+)\s*;", block)
        sf = re.search(r"\bstartFace\s+(\d+)\s*;", block)
        if not nf or not sf:
            raise ValueError(f"{path}: patch {name} lacks nFaces/startFace")
        patches.append((name, int(nf.group(1)), int(sf.group(1))))
    if len(patches) != n:
        raise ValueError(f"{path}: expected {n} patches, found {len(patches)}")
    return patches


def read_polymesh(path: str, scale: float = 1.0) -> PolyMesh:
    """Read an ASCII OpenFOAM polyMesh directory (points scaled by ``scale``)."""
    points = _read_points(os.path.join(path, "points"), scale)
    offsets, nodes = _read_faces(os.path.join(path, "faces"))
    owner = _read_labels(os.path.join(path, "owner"))
    neighbour = _read_labels(os.path.join(path, "neighbour"))
    patches = _read_boundary(os.path.join(path, "boundary"))
    nf = offsets.size - 1
    if owner.size != nf:
        raise ValueError(f"{path}: {owner.size} owners for {nf} faces")
    start = neighbour.size
    for name, n, s in patches:
        if s != start:
            raise ValueError(f"{path}: patch {name} starts at face {s}, expected {start} (patches must be "
                             f"contiguous after the internal faces)")
        start += n
    if start != nf:
        raise ValueError(f"{path}: patches cover faces up to {start}, the mesh has {nf}")
    return PolyMesh(points=points, face_offsets=offsets, face_nodes=nodes, owner=owner, neighbour=neighbour,
                    patch_names=[p[0] for p in patches], patch_sizes=[p[1] for p in patches])


def FOAM3D_mesh(path: str, scale: float = 1.0, device: int | None = None) -> Mesh3:
    """FOAM3D_mesh(meshFile; scale) (src/FoamMesh/FoamMesh_5_build.jl:21-27):
    read a polyMesh directory and build the Mesh3 (Float64, 0-based); with
    ``device`` the geometry is computed on that GPU."""
    return build_mesh3(read_polymesh(path, scale), device=device)


_HEADER = """/*--------------------------------*- C++ -*----------------------------------*\\
  written by xcalibre_b200
\\*---------------------------------------------------------------------------*/
FoamFile
{{
    format      ascii;
    class       {cls};
    location    "constant/polyMesh";
    object      {obj};
}}
// * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * //

"""


def write_polymesh(pm: PolyMesh, path: str) -> None:
    """Write ``pm`` as an ASCII polyMesh directory (points with 17
    significant digits, so reading them back gives the same doubles)."""
    os.makedirs(path, exist_ok=True)
    pts = np.asarray(pm.points, dtype=np.float64)
    with open(os.path.join(path, "points"), "w") as f:
        f.write(_HEADER.format(cls="vectorField", obj="points"))
        f.write(f"{pts.shape[0]}\n(\n")
        f.write("".join(f"({x!r} {y!r} {z!r})\n" for x, y, z in pts.tolist()))
        f.write(")\n")
    off = np.asarray(pm.face_offsets)
    nodes = np.asarray(pm.face_nodes)
    with open(os.path.join(path, "faces"), "w") as f:
        f.write(_HEADER.format(cls="faceList", obj="faces"))
        f.write(f"{off.size - 1}\n(\n")
        f.write("".join(f"{off[k + 1] - off[k]}({' '.join(map(str, nodes[off[k]:off[k + 1]].tolist()))})\n"
                        for k in range(off.size - 1)))
        f.write(")\n")
    for name, arr in (("owner", pm.owner), ("neighbour", pm.neighbour)):
        a = np.asarray(arr)
        with open(os.path.join(path, name), "w") as f:
            f.write(_HEADER.format(cls="labelList", obj=name))
            f.write(f"{a.size}\n(\n")
            f.write("\n".join(map(str, a.tolist())))
            f.write("\n)\n")
    with open(os.path.join(path, "boundary"), "w") as f:
        f.write(_HEADER.format(cls="polyBoundaryMesh", obj="boundary"))
        f.write(f"{len(pm.patch_sizes)}\n(\n")
        start = int(np.asarray(pm.neighbour).size)
        for name, n in zip(pm.patch_names, pm.patch_sizes):
            f.write(f"    {name}\n    {{\n        type            patch;\n        nFaces          {int(n)};\n"
                    f"        startFace       {start};\n    }}\n")
            start += int(n)
        f.write(")\n")
