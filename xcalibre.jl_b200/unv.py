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
                 patch_count=patch_count, points=points, dim=2, cell_nodes=[list(vs) for vs in cells_nodes])


# ---------------------------------------------------------------------------
# 3D meshes: UNV3D_mesh (src/UNV3)
# ---------------------------------------------------------------------------
def _unv_float(s: str) -> float:
    """_parse_unv_float (UNV3_1_reader.jl:150-156): Fortran 'D' exponents."""
    return float(s.replace("D", "e").replace("d", "e"))


def read_unv3(path: str, scale: float = 1.0):
    """read_UNV3 (UNV3_1_reader.jl:12-148): (points [n, 3] scaled, faces
    [vertex lists, 0-based], cells [vertex lists, 0-based], groups [(name,
    [face positions, 1-based])]).  After each "-1" the next line names the
    dataset; 2411 points are its 3-field lines; 2412 elements are 6-field
    headers (edges: type 11 or 2 nodes, one line skipped; faces: 41 with 3
    or 44 with 4 nodes; cells: 111, 112, 115, nodes over as many lines as
    needed), numbered edges, then faces, then cells; 2467 groups are a name
    line then 8- or 4-field entity lines whose element labels (fields 2 and
    6) less the edge count are face positions."""
    points, faces, cells, groups = [], [], [], []
    n_edge = 0
    with open(path, "r") as f:
        lines = iter(f)
        ds = ""
        for line in lines:
            line = line.strip()
            if not line:
                continue
            if line == "-1":
                if ds == "":
                    ds = next(lines).strip()
                    if ds == "-1":
                        ds = ""
                else:
                    ds = ""
                continue
            t = line.split()
            if ds == "2411":
                if len(t) == 3:
                    points.append((_unv_float(t[0]) * scale, _unv_float(t[1]) * scale, _unv_float(t[2]) * scale))
            elif ds == "2412":
                if len(t) != 6:
                    continue
                eid, etype, nn = int(t[0]), int(t[1]), int(t[5])
                if nn == 2 or etype == 11:
                    n_edge += 1
                    next(lines)
                elif (etype == 41 and nn == 3) or (etype == 44 and nn == 4):
                    if eid - n_edge != len(faces) + 1:
                        raise ValueError(f"{path}: face index in UNV file are not in order at UNV index {eid}")
                    faces.append([int(v) - 1 for v in next(lines).split()])
                elif etype in (111, 115, 112):
                    if eid - len(faces) - n_edge != len(cells) + 1:
                        raise ValueError(f"{path}: cell index in UNV file are not in order at UNV index {eid}")
                    nodes = []
                    while len(nodes) < nn:
                        nodes.extend(int(v) - 1 for v in next(lines).split())
                    cells.append(nodes)
            elif ds == "2467":
                if len(t) == 1 and _try_int(t[0]) is None:
                    groups.append((t[0], []))
                elif groups:
                    if len(t) == 8 and int(t[1]) != 0:
                        groups[-1][1].extend((int(t[1]) - n_edge, int(t[5]) - n_edge))
                    elif len(t) == 4 and int(t[1]) != 0:
                        groups[-1][1].append(int(t[1]) - n_edge)
    return np.array(points, dtype=np.float64).reshape(-1, 3), faces, cells, groups


_TET = ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3))
_HEX = ((0, 1, 2, 3), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7))
_PRI3 = ((0, 1, 2), (3, 4, 5))
_PRI4 = ((0, 1, 4, 3), (1, 2, 5, 4), (2, 0, 3, 5))


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def UNV3D_mesh(path: str, scale: float = 1.0) -> Mesh3:
    """UNV3D_mesh(meshFile; scale) (UNV3_2_builder.jl:14-30)."""
    return unv3_mesh(*read_unv3(path, scale), source=path)


def _unv3_polymesh(points, fnodes, owner, neigh, nB, groups):
    """The polyMesh view of a UNV3 mesh, for the result writers: internal
    faces first, each with the lower-numbered cell as owner (its nodes
    reversed when that swaps owner and neighbour, so the normal keeps
    pointing out of the owner), in (owner, neighbour) order; then the
    boundary faces, group by group.  fnodes are oriented out of their owner
    (as calculate_face_properties! leaves them)."""
    from .meshgen import PolyMesh
    internal = []
    for f in range(nB, len(fnodes)):
        o, n, fn = owner[f], neigh[f], list(fnodes[f])
        if o > n:
            o, n, fn = n, o, fn[::-1]
        internal.append((o, n, fn))
    internal.sort(key=lambda t: (t[0], t[1]))
    faces = [t[2] for t in internal] + [list(fnodes[f]) for f in range(nB)]
    off = np.zeros(len(faces) + 1, dtype=np.int32)
    off[1:] = np.cumsum([len(fn) for fn in faces])
    return PolyMesh(points=np.asarray(points, dtype=np.float64), face_offsets=off,
                    face_nodes=np.array([v for fn in faces for v in fn], dtype=np.int32),
                    owner=np.array([t[0] for t in internal] + [owner[f] for f in range(nB)], dtype=np.int32),
                    neighbour=np.array([t[1] for t in internal], dtype=np.int32),
                    patch_names=[g[0] for g in groups], patch_sizes=[len(g[1]) for g in groups])


def unv3_mesh(points, faces, cells, groups, source: str = "mesh") -> Mesh3:
    """_build_UNV3D_mesh_core (UNV3_2_builder.jl:32-64): boundary faces in
    group order, each owned by the first cell (of its first node's cells)
    holding all its nodes; internal faces from each cell's element faces
    (tet, hex, prism maps; a face keyed by its sorted nodes, boundary keys
    skipped), owner the first cell to list it and neighbour the second;
    then calculate_centres! (node means), calculate_face_properties! (a
    triangle fan about the face's node mean: area vector, fan-weighted
    centroid, normal = area vector / (area + 1e-16), oriented out of the
    owner, weight/delta/e from the node-mean cell centres) and
    calculate_area_and_volume! (pyramids on each face from the node-mean
    centre: volume sum and volume-weighted centroid)."""
    pts = [tuple(p) for p in np.asarray(points, dtype=np.float64).tolist()]
    nC = len(cells)
    node_cells = [[] for _ in pts]
    for c, vs in enumerate(cells):
        for v in vs:
            node_cells[v].append(c)
    b_nodes, b_cell, bkeys = [], [], {}
    for name, fl in groups:
        for fi in fl:
            nodes = faces[fi - 1]
            owner = -1
            for c in node_cells[nodes[0]]:
                if all(n in cells[c] for n in nodes):
                    owner = c
                    break
            if owner < 0:
                raise ValueError(f"{source}: boundary face {fi} has no cell")
            bkeys[tuple(sorted(nodes))] = len(b_nodes)
            b_nodes.append(list(nodes))
            b_cell.append(owner)
    nB = len(b_nodes)
    i_nodes, i_own, ikeys = [], [], {}
    for c, vs in enumerate(cells):
        nc = len(vs)
        maps = _TET if nc == 4 else (_PRI3 + _PRI4 if nc == 6 else (_HEX if nc == 8 else ()))
        for mp in maps:
            fn = [vs[q] for q in mp]
            key = tuple(sorted(fn))
            if key in bkeys:
                continue
            k = ikeys.get(key)
            if k is not None:
                i_own[k][1] = c
            else:
                ikeys[key] = len(i_nodes)
                i_nodes.append(fn)
                i_own.append([c, -1])
    if any(o[1] < 0 for o in i_own):
        raise ValueError(f"{source}: an internal face has one cell")
    fnodes = b_nodes + i_nodes
    owner = b_cell + [o[0] for o in i_own]
    neigh = b_cell + [o[1] for o in i_own]
    nF = len(fnodes)
    c_faces = [[] for _ in range(nC)]
    c_sign = [[] for _ in range(nC)]
    c_nb = [[] for _ in range(nC)]
    for f in range(nB, nF):
        o, n = owner[f], neigh[f]
        c_faces[o].append(f)
        c_sign[o].append(1)
        c_nb[o].append(n)
        c_faces[n].append(f)
        c_sign[n].append(-1)
        c_nb[n].append(o)
    cc = [_mean(pts, vs) for vs in cells]  # calculate_centres!
    fc0 = [_mean(pts, fn) for fn in fnodes]
    fc = [None] * nF
    normal = [None] * nF
    area = [0.0] * nF
    e_vec = [None] * nF
    delta = [0.0] * nF
    weight = [0.0] * nF
    for f in range(nF):  # calculate_face_properties!
        fn = fnodes[f]
        L = len(fn)
        C1 = cc[owner[f]]
        E = fc0[f]
        ax = ay = az = 0.0
        tx = ty = tz = 0.0
        sa = 0.0
        for j in range(L):
            p1, p2 = pts[fn[j]], pts[fn[(j + 1) % L]]
            cr = _cross(_sub(p1, E), _sub(p2, E))
            a = (0.5 * cr[0], 0.5 * cr[1], 0.5 * cr[2])
            am = _norm(a)
            ax, ay, az = ax + a[0], ay + a[1], az + a[2]
            sa = sa + am
            m3 = ((E[0] + p1[0]) + p2[0], (E[1] + p1[1]) + p2[1], (E[2] + p1[2]) + p2[2])
            tx, ty, tz = tx + am * (m3[0] / 3.0), ty + am * (m3[1] / 3.0), tz + am * (m3[2] / 3.0)
        av = (ax, ay, az)
        A = _norm(av)
        n = _div(av, A + 1e-16)
        F = _div((tx, ty, tz), sa + 1e-16)
        check = _sub(F, C1) if f < nB else _sub(cc[neigh[f]], C1)
        if _dot(check, n) < 0.0:
            n = _neg(n)
            fnodes[f] = fn[::-1] if L > 1 else fn
        if f < nB:
            weight[f], delta[f], e_vec[f] = _wde_boundary(_sub(F, C1), n)
        else:
            C2 = cc[neigh[f]]
            weight[f], delta[f], e_vec[f] = _wde_internal(_sub(F, C1), _sub(F, C2), _sub(C2, C1), n)
        fc[f], normal[f], area[f] = F, n, A
    # calculate_area_and_volume!: per cell its boundary faces, then its
    # internal faces, each in face order
    per = [[] for _ in range(nC)]
    for f in range(nB):
        per[b_cell[f]].append(f)
    for f in range(nB, nF):
        per[owner[f]].append(f)
        per[neigh[f]].append(f)
    centre = [None] * nC
    volume = [0.0] * nC
    third = 1.0 / 3.0
    for c in range(nC):
        apex = cc[c]
        vt = 0.0
        qx = qy = qz = 0.0
        for f in per[c]:
            h = _sub(fc[f], apex)
            S = (normal[f][0] * area[f], normal[f][1] * area[f], normal[f][2] * area[f])
            if _dot(h, S) < 0.0:
                S = _neg(S)
            vp = third * _dot(h, S)
            Cp = (0.75 * fc[f][0] + 0.25 * apex[0], 0.75 * fc[f][1] + 0.25 * apex[1], 0.75 * fc[f][2] + 0.25 * apex[2])
            vt = vt + vp
            qx, qy, qz = qx + vp * Cp[0], qy + vp * Cp[1], qz + vp * Cp[2]
        volume[c] = abs(vt)
        centre[c] = _div((qx, qy, qz), vt) if vt > 1e-16 else apex
    patch_count, patch_start, s = [], [], 0
    for _, fl in groups:
        patch_start.append(s)
        patch_count.append(len(fl))
        s += len(fl)
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
                 cell_faces_offset=off, cell_faces=cat(c_faces), cell_nsign=cat(c_sign), cell_neighbours=cat(c_nb),
                 boundary_cellsID=np.array(b_cell, dtype=np.int32), patch_names=[g[0] for g in groups],
                 patch_start=np.array(patch_start, dtype=np.int32), patch_count=np.array(patch_count, dtype=np.int32),
                 points=np.asarray(points, dtype=np.float64), dim=3,
                 polymesh=_unv3_polymesh(points, fnodes, owner, neigh, nB, groups))
