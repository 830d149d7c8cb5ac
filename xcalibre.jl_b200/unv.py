"""I-DEAS universal (.unv) mesh files -> Mesh3 (0-based, Float64).

``UNV2D_mesh`` restates src/UNV2 (XCALibre's 2D reader and builder):

* ``read_unv2`` (UNV2_1_loader.jl:1-120) walks the file's line blocks:
  dataset 2411 gives the points (lines whose first field holds a '.'),
  dataset 2412 the elements (a 6-field header whose last field is the vertex
  count 2, 3 or 4, then the vertex line; the beam orientation line "0 ..."
  is skipped), dataset 2467 the groups (a header "<n> 0 ...", a name line,
  then entity lines whose fields 2 and 6 are element positions);
* ``generate``/``connect!`` (UNV2_3_builder.jl:32-253): boundary faces first,
  one per group element in group order, then each cell's edges (each face
  stored as its sorted vertex pair; later duplicates dropped); a face's
  owner and neighbour are the cells shared by both its nodes, in cell
  order; a group's faces are the first boundary faces whose vertex pair
  matches its element's two smallest vertices;
* ``process_geometry!`` (UNV2_2_geometry.jl:1-260): node-mean centres for
  cells and faces; per face the edge length as area and the in-plane normal
  tangent x (0,0,1), oriented from owner to neighbour (boundary faces: out
  of the owner); weight, delta and e from ``weight_delta_e``
  (Mesh_1_functions.jl:20-51) with the node-mean cell centres; then each
  cell's centre becomes the area-weighted mean of its face centres, its
  sign per internal face the sign of (face centre - centre).normal, and its
  area 0.5 sum (d.n s) A_f.

Arithmetic runs in the reference's operation order on Python floats (IEEE
double, no fused multiply-add).  The result is a Mesh3 with ``dim = 2``:
the finite-volume path treats it like any mesh (its z momentum has a zero
right-hand side, so U_z stays 0 with a zero residual, as the reference's
skipped z solve gives); what differs for a 2D mesh (the Courant cell size
sqrt(V), the LES filter scaling (1, 0.5)) keys on ``dim``.
"""
from __future__ import annotations

import math

import numpy as np

from .foam import Mesh3

_EPS1 = float(np.spacing(1.0))


def _try_int(s: str):
    try:
        return int(s)
    except ValueError:
        return None


def read_unv2(path: str):
    """(points [n, 3], elements [(index, vertex count, vertices 0-based)],
    groups [(name, [element positions, 1-based])]) of a 2D .unv file."""
    points, elements, groups = [], [], []
    block = False
    ds = None
    index = count = 0
    with open(path, "r") as f:
        for line in f:
            s = line.split()
            if not s:
                continue
            if s[0] == "-1":
                block = not block
                ds = None
                continue
            if block and ds is None and s[0] in ("2411", "2412", "2467"):
                ds = s[0]
                continue
            if ds == "2411":
                if "." in s[0]:
                    points.append((float(s[0]), float(s[1]), float(s[2])))
                continue
            if ds == "2412":
                if int(s[0]) == 0:
                    continue
                if len(s) == 6 and int(s[-1]) in (2, 3, 4):
                    count, index = int(s[-1]), int(s[0])
                    continue
                if len(s) in (2, 3, 4):
                    elements.append((index, count, [int(v) - 1 for v in s]))
                continue
            if ds == "2467":
                if _try_int(s[0]) is not None and len(s) > 1 and _try_int(s[1]) == 0:
                    groups.append(["default", []])
                    continue
                if _try_int(s[0]) is None:
                    groups[-1][0] = s[0]
                    continue
                groups[-1][1].append(int(s[1]))
                if len(s) >= 6:
                    groups[-1][1].append(int(s[5]))
    return np.array(points, dtype=np.float64).reshape(-1, 3), elements, [(n, e) for n, e in groups]


def _sub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _norm(a):
    return math.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])


def _div(a, s):
    return (a[0] / s, a[1] / s, a[2] / s)


def _neg(a):
    return (-a[0], -a[1], -a[2])


def _eps(x):
    return float(np.spacing(abs(x)))


def _mean(pts, ids):
    sx = sy = sz = 0.0
    for i in ids:
        p = pts[i]
        sx, sy, sz = sx + p[0], sy + p[1], sz + p[2]
    n = float(len(ids))
    return (sx / n, sy / n, sz / n)


def _normal2d(t):
    # unit_tangent x SVector(0, 0, 1)
    return (t[1] * 1.0 - t[2] * 0.0, t[2] * 0.0 - t[0] * 1.0, t[0] * 0.0 - t[1] * 0.0)


def _wde_internal(C1F1, C2F1, C1C2, n):
    """weight_delta_e(C1F1, C2F1, C1C2, normal) (Mesh_1_functions.jl:20-42)."""
    projection = _dot(C1C2, n)
    if math.isfinite(projection) and abs(projection) > _eps(projection):
        weight = 1.0 - _dot(C1F1, n) / projection
    else:
        d1, d2 = _norm(C1F1), _norm(C2F1)
        dsum = d1 + d2
        weight = d2 / dsum if dsum > 0.0 else 0.5
    delta = _norm(C1C2)
    if delta > 0.0:
        e = _div(C1C2, delta)
    else:
        delta = _norm(C1F1) + _norm(C2F1)
        e = n
    delta = max(delta, _EPS1)
    weight = min(max(weight, 0.0), 1.0)
    return weight, delta, e


def _wde_boundary(C1F1, n):
    """weight_delta_e(C1F1, normal) (Mesh_1_functions.jl:45-51)."""
    delta = _norm(C1F1)
    e = _div(C1F1, delta) if delta > 0.0 else n
    return 1.0, max(delta, _EPS1), e


def UNV2D_mesh(path: str, scale: float = 1.0) -> Mesh3:
    """UNV2D_mesh(meshFile; scale) (UNV2_3_builder.jl:11-55): read a 2D .unv
    file and build its mesh (points multiplied by ``scale``)."""
    return unv2_mesh(*read_unv2(path), scale=scale, source=path)


def unv2_mesh(points, elements, groups, scale: float = 1.0, source: str = "mesh") -> Mesh3:
    """The mesh of already-read UNV data: ``points`` [n, 3], ``elements``
    [(index, vertex count, vertices 0-based)], ``groups`` [(name, [element
    positions, 1-based])]."""
    points = np.asarray(points, dtype=np.float64)
    if scale != 1:
        points = points * scale
    pts = [tuple(p) for p in points.tolist()]
    first = next((k for k, e in enumerate(elements) if e[1] > 2), None)
    if first is None:
        raise ValueError(f"{source}: no 2D elements")
    cells_nodes = [e[2] for e in elements[first:]]
    nC = len(cells_nodes)
    node_cells = [[] for _ in pts]
    for c, vs in enumerate(cells_nodes):
        for v in vs:
            node_cells[v].append(c)

    def edge(a, b):
        if a == b:
            raise ValueError("Boundary elements are inconsistent: possible mesh corruption")
        return (a, b) if a < b else (b, a)

    nbf = sum(len(g[1]) for g in groups)
    raw = [edge(elements[e - 1][2][0], elements[e - 1][2][1]) for _, els in groups for e in els]
    for vs in cells_nodes:
        n = len(vs)
        raw.extend(edge(vs[i], vs[(i + 1) % n]) for i in range(n))
    faces = list(dict.fromkeys(raw))  # unique!: first occurrences, in order
    nF = len(faces)

    owner = [0] * nF
    neigh = [0] * nF
    c_faces = [[] for _ in range(nC)]
    c_neigh = [[] for _ in range(nC)]
    for f, (n1, n2) in enumerate(faces):
        own = [c1 for c1 in node_cells[n1] for c2 in node_cells[n2] if c1 == c2]
        if len(own) > 2 or not own:
            raise ValueError(f"{source}: face {f} is shared by {len(own)} cells")
        if len(own) == 2:
            owner[f], neigh[f] = own
            c_faces[own[0]].append(f)
            c_faces[own[1]].append(f)
            c_neigh[own[0]].append(own[1])
            c_neigh[own[1]].append(own[0])
        else:
            owner[f] = neigh[f] = own[0]

    first_b = {}
    for f in range(nbf):
        first_b.setdefault(faces[f], []).append(f)
    b_faces, b_cells = [], []
    for _, els in groups:
        fl, cl = [], []
        for e in els:
            key = tuple(sorted(elements[e - 1][2])[:2])
            for f in first_b.get(key, []):
                fl.append(f)
                cl.append(owner[f])
        b_faces.append(fl)
        b_cells.append(cl)
    nB = sum(len(fl) for fl in b_faces)

    cc = [_mean(pts, vs) for vs in cells_nodes]
    fc = [_mean(pts, fn) for fn in faces]
    area = [0.0] * nF
    normal = [(0.0, 0.0, 0.0)] * nF
    e_vec = [(0.0, 0.0, 0.0)] * nF
    delta = [0.0] * nF
    weight = [0.0] * nF
    for f in range(nB, nF):  # internal_face_properties!
        n1, n2 = faces[f]
        tangent = _sub(pts[n2], pts[n1])
        a = _norm(tangent)
        C1, C2 = cc[owner[f]], cc[neigh[f]]
        C1F1, C2F1, C1C2 = _sub(fc[f], C1), _sub(fc[f], C2), _sub(C2, C1)
        n = _normal2d(_div(tangent, a))
        if _dot(C1C2, n) < 0.0:
            n = _neg(n)
        weight[f], delta[f], e_vec[f] = _wde_internal(C1F1, C2F1, C1C2, n)
        area[f], normal[f] = a, n
    for fl in b_faces:  # boundary_face_properties!
        for f in fl:
            n1, n2 = faces[f]
            tangent = _sub(pts[n2], pts[n1])
            a = _norm(tangent)
            n = _normal2d(_div(tangent, a))
            C1F1 = _sub(fc[f], cc[owner[f]])
            if _dot(C1F1, n) < 0.0:
                n = _neg(n)
            weight[f], delta[f], e_vec[f] = _wde_boundary(C1F1, n)
            area[f], normal[f] = a, n

    all_faces = [list(fl) for fl in c_faces]  # cell_properties!
    for fl, cl in zip(b_faces, b_cells):
        for f, c in zip(fl, cl):
            all_faces[c].append(f)
    centre = [None] * nC
    volume = [0.0] * nC
    nsign = [[] for _ in range(nC)]
    for c in range(nC):
        sx = sy = sz = 0.0
        sa = 0.0
        for f in all_faces[c]:
            sx, sy, sz = sx + fc[f][0] * area[f], sy + fc[f][1] * area[f], sz + fc[f][2] * area[f]
            sa = sa + area[f]
        tc = (sx / sa, sy / sa, sz / sa)
        internal = set(c_faces[c])
        vol = 0.0
        for f in all_faces[c]:
            d = _dot(_sub(fc[f], tc), normal[f])
            s = 1 if d > 0.0 else -1
            if f in internal:
                nsign[c].append(s)
            vol = vol + (d * s) * area[f]
        centre[c] = tc
        volume[c] = 0.5 * vol

    bcell = np.zeros(nB, dtype=np.int32)
    for fl, cl in zip(b_faces, b_cells):
        bcell[fl] = cl
    patch_start = np.array([min(fl) for fl in b_faces], dtype=np.int32)
    patch_count = np.array([max(fl) - min(fl) + 1 for fl in b_faces], dtype=np.int32)
    off = np.zeros(nC + 1, dtype=np.int32)
    off[1:] = np.cumsum([len(v) for v in c_faces])

    def cat(lists):
        return np.array([v for lst in lists for v in lst], dtype=np.int32)

    return Mesh3(n_cells=nC, n_faces=nF, n_bfaces=nB,
                 face_owner=np.array(owner, dtype=np.int32), face_neigh=np.array(neigh, dtype=np.int32),
                 face_centre=np.array(fc, dtype=np.float64), face_normal=np.array(normal, dtype=np.float64),
                 face_e=np.array(e_vec, dtype=np.float64), face_area=np.array(area, dtype=np.float64),
                 face_delta=np.array(delta, dtype=np.float64), face_weight=np.array(weight, dtype=np.float64),
                 cell_centre=np.array(centre, dtype=np.float64), cell_volume=np.array(volume, dtype=np.float64),
                 cell_faces_offset=off, cell_faces=cat(c_faces), cell_nsign=cat(nsign), cell_neighbours=cat(c_neigh),
                 boundary_cellsID=bcell, patch_names=[g[0] for g in groups], patch_start=patch_start,
                 patch_count=patch_count, points=points, dim=2)
