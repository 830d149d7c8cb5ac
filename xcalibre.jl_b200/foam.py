"""Mesh3 construction from a polyMesh (host side, once per mesh).

This is the product's import of a polyMesh into the Mesh3 contract consumed by
``xcal_mesh_upload``.  It restates XCALibre's ``FOAM3D_mesh`` pipeline with
vectorised numpy, keeping every floating-point operation in the order the
Julia source writes it (numpy performs each elementwise op as one IEEE
rounding, so the result is bit-identical to a scalar loop):

  src/FoamMesh/FoamMesh_1_read.jl:25-43     assign_faces!
  src/FoamMesh/FoamMesh_2_connect.jl:24-69  connect_cell_faces
  src/FoamMesh/FoamMesh_2_connect.jl:71-146 connect_cell_nodes
  src/FoamMesh/FoamMesh_2_connect.jl:148-195 connect_face_nodes
  src/FoamMesh/FoamMesh_3_generate.jl:2-82  generate_mesh
  src/FoamMesh/FoamMesh_4_geometry.jl:2-158 compute_geometry!
  src/Mesh/Mesh_1_functions.jl:20-51        weight_delta_e

Indices are 0-based; faces 0..n_bfaces-1 are the boundary faces.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .meshgen import PolyMesh

_EPS1 = np.spacing(1.0)  # Julia eps(1.0)


@dataclass
class Mesh3:
    n_cells: int
    n_faces: int
    n_bfaces: int
    face_owner: np.ndarray       # int32 [n_faces]
    face_neigh: np.ndarray       # int32 [n_faces]
    face_centre: np.ndarray      # float64 [n_faces, 3]
    face_normal: np.ndarray      # float64 [n_faces, 3]
    face_e: np.ndarray           # float64 [n_faces, 3]
    face_area: np.ndarray        # float64 [n_faces]
    face_delta: np.ndarray       # float64 [n_faces]
    face_weight: np.ndarray      # float64 [n_faces]
    cell_centre: np.ndarray      # float64 [n_cells, 3]
    cell_volume: np.ndarray      # float64 [n_cells]
    cell_faces_offset: np.ndarray  # int32 [n_cells+1]
    cell_faces: np.ndarray       # int32 [2*n_ifaces]
    cell_nsign: np.ndarray       # int32 [2*n_ifaces]
    cell_neighbours: np.ndarray  # int32 [2*n_ifaces]
    boundary_cellsID: np.ndarray  # int32 [n_bfaces]
    patch_names: list
    patch_start: np.ndarray      # int32 [n_patches]
    patch_count: np.ndarray      # int32 [n_patches]
    points: np.ndarray | None = None
    face_nodes_offset: np.ndarray | None = None
    face_nodes: np.ndarray | None = None

    @property
    def n_ifaces(self) -> int:
        return self.n_faces - self.n_bfaces

    def patch_index(self, name: str) -> int:
        try:
            return self.patch_names.index(name)
        except ValueError:
            raise KeyError(f'"{name}" is not a recognised boundary name') from None

    def patch_range(self, name: str) -> range:
        p = self.patch_index(name)
        s = int(self.patch_start[p])
        return range(s, s + int(self.patch_count[p]))

    def __repr__(self) -> str:  # Base.show(io, mesh) (Mesh_0_types.jl:185-198)
        n_nodes = 0 if self.points is None else len(self.points)
        return f"3D Mesh with:\n-> {self.n_cells} cells\n-> {self.n_faces} faces\n-> {n_nodes} nodes"


def _norm(v):
    # norm(SVector) = sqrt((x^2 + y^2) + z^2)
    return np.sqrt(v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1] + v[..., 2] * v[..., 2])


def _dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def _grouped_sequential_sum(values, offsets):
    """Per-group sequential sum of ``values`` (rows) grouped by CSR offsets,
    starting from 0.0 and adding in order (a scalar loop's rounding)."""
    counts = np.diff(offsets)
    n = counts.shape[0]
    out = np.zeros((n,) + values.shape[1:], dtype=np.float64)
    maxc = int(counts.max()) if n else 0
    for k in range(maxc):
        sel = counts > k
        idx = offsets[:-1][sel] + k
        out[sel] = out[sel] + values[idx]
    return out


def build_mesh3(pm: PolyMesh) -> Mesh3:
    """FOAM3D_mesh restatement: polyMesh -> Mesh3 (Float64, 0-based)."""
    n_faces = pm.n_faces
    n_if = pm.n_internal_faces
    n_bf = n_faces - n_if
    n_cells = pm.n_cells
    owner = pm.owner.astype(np.int64)
    neigh_foam = np.concatenate([pm.neighbour.astype(np.int64), owner[n_if:]])  # assign_faces!

    # connect_cell_faces: entries (cell, fID, sign, other) in increasing fi,
    # owner entry before neighbour entry; stable sort by cell keeps that order.
    fi = np.arange(n_if, dtype=np.int64)
    cells_il = np.empty(2 * n_if, dtype=np.int64)
    cells_il[0::2] = owner[:n_if]
    cells_il[1::2] = neigh_foam[:n_if]
    fid_il = np.repeat(fi + n_bf, 2)
    sign_il = np.tile(np.array([1, -1], dtype=np.int64), n_if)
    other_il = np.empty(2 * n_if, dtype=np.int64)
    other_il[0::2] = neigh_foam[:n_if]
    other_il[1::2] = owner[:n_if]
    order = np.argsort(cells_il, kind="stable")
    cell_faces = fid_il[order]
    cell_nsign = sign_il[order]
    cell_neigh = other_il[order]
    cf_off = np.zeros(n_cells + 1, dtype=np.int64)
    np.cumsum(np.bincount(cells_il, minlength=n_cells), out=cf_off[1:])

    # connect_cell_nodes: raw list per cell (owner role then neighbour role per
    # face, foam face order), first-seen dedup
    fo = pm.face_offsets.astype(np.int64)
    fsz = np.diff(fo)
    fn = pm.face_nodes.astype(np.int64)
    # Per cell, the raw node list is the node lists of its faces in foam face
    # order (a boundary face's second, neighbour-role copy repeats nodes just
    # added and is dropped by the dedup, so it is skipped here).  Dedup keeps
    # first occurrences.  Done densely: one row per cell.
    fcell = np.concatenate([owner, neigh_foam[:n_if]])
    fidx = np.concatenate([np.arange(n_faces), np.arange(n_if)])
    o = np.argsort(fcell * (n_faces + 1) + fidx, kind="stable")
    fcell, fidx = fcell[o], fidx[o]
    cf_cnt = np.bincount(fcell, minlength=n_cells)
    cf_start = np.zeros(n_cells + 1, dtype=np.int64)
    np.cumsum(cf_cnt, out=cf_start[1:])
    pos = np.arange(fcell.shape[0]) - cf_start[fcell]      # face slot within its cell
    node_cnt = np.zeros(n_cells, dtype=np.int64)
    np.add.at(node_cnt, fcell, fsz[fidx])
    maxraw = int(node_cnt.max())
    # column offset of each (cell, face) entry inside the cell's row
    col0 = np.zeros(fcell.shape[0], dtype=np.int64)
    maxf = int(cf_cnt.max())
    run = np.zeros(n_cells, dtype=np.int64)
    for k in range(maxf):
        sel = np.nonzero(pos == k)[0]
        col0[sel] = run[fcell[sel]]
        run[fcell[sel]] += fsz[fidx[sel]]
    R = np.full((n_cells, maxraw), -1, dtype=np.int64)
    maxn = int(fsz.max())
    for j in range(maxn):
        sel = np.nonzero(fsz[fidx] > j)[0]
        R[fcell[sel], col0[sel] + j] = fn[fo[fidx[sel]] + j]
    keep = R >= 0
    for j in range(1, maxraw):
        col = R[:, j]
        dup = np.zeros(n_cells, dtype=bool)
        for i in range(j):
            dup |= (R[:, i] == col)
        keep[:, j] &= ~dup
    cn_node = R[keep]                                      # row-major: cell order, first-seen order
    cn_cell = np.nonzero(keep)[0]
    cn_off = np.zeros(n_cells + 1, dtype=np.int64)
    np.cumsum(np.bincount(cn_cell, minlength=n_cells), out=cn_off[1:])
    del R, keep

    # connect_face_nodes: boundary faces first, then internal faces
    src = np.concatenate([np.arange(n_if, n_faces), np.arange(n_if)])
    m_fsz = fsz[src]
    m_fo = np.zeros(n_faces + 1, dtype=np.int64)
    np.cumsum(m_fsz, out=m_fo[1:])
    m_fn = _gather_ranges(fn, fo[src], m_fsz)

    f_owner = owner[src]
    f_neigh = neigh_foam[src]
    bcell = f_owner[:n_bf]

    pts = pm.points.astype(np.float64)
    # calculate_cell_centres! / calculate_face_centres!
    ccentre = _grouped_sequential_sum(pts[cn_node], cn_off) / np.diff(cn_off).astype(np.float64)[:, None]
    fcentre0 = _grouped_sequential_sum(pts[m_fn], m_fo) / m_fsz.astype(np.float64)[:, None]

    # _face_geometry (fan triangles about the node-average apex)
    area_vec = np.zeros((n_faces, 3))
    centre_sum = np.zeros((n_faces, 3))
    sum_area = np.zeros(n_faces)
    maxn = int(m_fsz.max())
    for i in range(maxn):
        sel = np.nonzero(m_fsz > i)[0]
        n_s = m_fsz[sel]
        j = np.where(i == n_s - 1, 0, i + 1)
        p1 = pts[m_fn[m_fo[sel] + i]]
        p2 = pts[m_fn[m_fo[sel] + j]]
        apex = fcentre0[sel]
        tri_vec = _cross(p1 - apex, p2 - apex) / 2.0
        tri_area = _norm(tri_vec)
        ok = tri_area > 0.0
        s2 = sel[ok]
        area_vec[s2] = area_vec[s2] + tri_vec[ok]
        centre_sum[s2] = centre_sum[s2] + (tri_area[ok][:, None] * ((apex[ok] + p1[ok]) + p2[ok])) / 3.0
        sum_area[s2] = sum_area[s2] + tri_area[ok]
    mag = _norm(area_vec)
    with np.errstate(invalid="ignore", divide="ignore"):
        normal = np.where((mag > 0.0)[:, None], area_vec / mag[:, None], 0.0)
        fcentre = np.where((sum_area > 0.0)[:, None], centre_sum / sum_area[:, None], fcentre0)

    weight = np.empty(n_faces)
    delta = np.empty(n_faces)
    e = np.empty((n_faces, 3))
    # boundary faces
    b = slice(0, n_bf)
    C1 = ccentre[f_owner[b]]
    C1F1 = fcentre[b] - C1
    flip = _dot(C1F1, normal[b]) < 0.0
    normal[b] = np.where(flip[:, None], -normal[b], normal[b])
    d = _norm(C1F1)
    with np.errstate(invalid="ignore", divide="ignore"):
        e[b] = np.where((d > 0.0)[:, None], C1F1 / d[:, None], normal[b])
    delta[b] = np.maximum(d, _EPS1)
    weight[b] = 1.0
    # internal faces
    it = slice(n_bf, n_faces)
    C1 = ccentre[f_owner[it]]
    C2 = ccentre[f_neigh[it]]
    C1F1 = fcentre[it] - C1
    C2F1 = fcentre[it] - C2
    C1C2 = C2 - C1
    flip = _dot(C1C2, normal[it]) < 0.0
    normal[it] = np.where(flip[:, None], -normal[it], normal[it])
    nrm = normal[it]
    projection = _dot(C1C2, nrm)
    good = np.isfinite(projection) & (np.abs(projection) > np.spacing(np.abs(projection)))
    with np.errstate(invalid="ignore", divide="ignore"):
        wi = _dot(C1F1, nrm) / projection
        w_a = 1.0 - wi
        d1 = _norm(C1F1)
        d2 = _norm(C2F1)
        dsum = d1 + d2
        w_b = np.where(dsum > 0.0, d2 / dsum, 0.5)
        w = np.where(good, w_a, w_b)
        dl = _norm(C1C2)
        e_it = np.where((dl > 0.0)[:, None], C1C2 / dl[:, None], nrm)
    dl = np.where(dl > 0.0, dl, d1 + d2)
    delta[it] = np.maximum(dl, _EPS1)
    weight[it] = np.where(w > 1.0, 1.0, np.where(w < 0.0, 0.0, w))
    e[it] = e_it

    # calculate_cell_volumes!: internal faces (cell_faces order), then boundary
    # faces in increasing face id
    oneThird = 1.0 / 3.0
    xf = fcentre[cell_faces] - ccentre[np.repeat(np.arange(n_cells), np.diff(cf_off))]
    contrib = ((oneThird * _dot(xf, normal[cell_faces])) * cell_nsign.astype(np.float64)) * mag[cell_faces]
    vol = _grouped_sequential_sum(contrib, cf_off)
    max_area = np.zeros(n_cells)
    np.maximum.at(max_area, np.repeat(np.arange(n_cells), np.diff(cf_off)), mag[cell_faces])
    # boundary faces: per cell in increasing face id
    if n_bf:
        xb = fcentre[:n_bf] - ccentre[bcell]
        cb = (oneThird * _dot(xb, normal[:n_bf])) * mag[:n_bf]
        ob = np.argsort(bcell, kind="stable")
        boff = np.zeros(n_cells + 1, dtype=np.int64)
        np.cumsum(np.bincount(bcell, minlength=n_cells), out=boff[1:])
        counts = np.diff(boff)
        for k in range(int(counts.max())):
            sel = np.nonzero(counts > k)[0]
            fids = ob[boff[sel] + k]
            vol[sel] = vol[sel] + cb[fids]
        np.maximum.at(max_area, bcell, mag[:n_bf])
    bad = ~(np.isfinite(vol) & (vol > 0.0))
    if bad.any():
        est = np.power(max_area[bad], 1.5) * 1e-3
        vb = vol[bad]
        vol[bad] = np.maximum(np.where(np.isfinite(vb), np.abs(vb), 0.0), est)

    patch_start = np.zeros(len(pm.patch_sizes), dtype=np.int32)
    if len(pm.patch_sizes):
        patch_start[1:] = np.cumsum(pm.patch_sizes)[:-1]
    if int(np.sum(pm.patch_sizes)) != n_bf:
        raise ValueError("patch face counts do not cover the boundary faces")
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    return Mesh3(
        n_cells=n_cells, n_faces=n_faces, n_bfaces=n_bf,
        face_owner=i32(f_owner), face_neigh=i32(f_neigh),
        face_centre=f64(fcentre), face_normal=f64(normal), face_e=f64(e),
        face_area=f64(mag), face_delta=f64(delta), face_weight=f64(weight),
        cell_centre=f64(ccentre), cell_volume=f64(vol),
        cell_faces_offset=i32(cf_off), cell_faces=i32(cell_faces), cell_nsign=i32(cell_nsign),
        cell_neighbours=i32(cell_neigh), boundary_cellsID=i32(bcell),
        patch_names=list(pm.patch_names), patch_start=patch_start,
        patch_count=np.asarray(pm.patch_sizes, dtype=np.int32),
        points=pts, face_nodes_offset=i32(m_fo), face_nodes=i32(m_fn))


def _gather_ranges(arr, starts, counts):
    """Concatenate arr[starts[i] : starts[i]+counts[i]] for all i."""
    total = int(counts.sum())
    offs = np.zeros(counts.shape[0] + 1, dtype=np.int64)
    np.cumsum(counts, out=offs[1:])
    idx = np.arange(total) - np.repeat(offs[:-1], counts) + np.repeat(starts, counts)
    return arr[idx]
