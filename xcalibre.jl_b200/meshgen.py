"""Synthetic OpenFOAM-style polyMesh generators for the benchmark cases.

A polyMesh here is the data an OpenFOAM ``constant/polyMesh`` directory holds
and that ``read_FOAM3D`` (src/FoamMesh/FoamMesh_1_read.jl:1-23) reads: points,
faces (node lists), owner, neighbour and the boundary patch list.  Internal
faces come first, then the patches' faces, patch by patch.  All indices are
0-based.

Generators:
  * :func:`box_polymesh` -- a structured hex box with named patches built from
    the six sides, optionally with cell and face numbering permuted from a seed
    (the unstructured gather pattern of the permuted-channel workload).
  * :func:`cavity_polymesh`, :func:`channel_polymesh`,
    :func:`periodic_box_polymesh` -- the lid-driven cavity slab, the 4x1x1
    channel and the periodic cube.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

SIDES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


@dataclass
class PolyMesh:
    points: np.ndarray            # (n_points, 3) float64
    face_offsets: np.ndarray      # (n_faces+1,) int32
    face_nodes: np.ndarray        # (sum of face sizes,) int32
    owner: np.ndarray             # (n_faces,) int32
    neighbour: np.ndarray         # (n_internal_faces,) int32
    patch_names: list = field(default_factory=list)
    patch_sizes: list = field(default_factory=list)

    @property
    def n_faces(self) -> int:
        return int(self.owner.shape[0])

    @property
    def n_internal_faces(self) -> int:
        return int(self.neighbour.shape[0])

    @property
    def n_cells(self) -> int:
        m = int(self.owner.max()) if self.owner.size else -1
        if self.neighbour.size:
            m = max(m, int(self.neighbour.max()))
        return m + 1


def box_polymesh(nx: int, ny: int, nz: int, lengths=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0),
                 patches=None, seed: int | None = None, skew: float = 0.0, skew_seed: int = 0) -> PolyMesh:
    """Hex box of nx*ny*nz cells on [origin, origin+lengths].

    ``patches`` is a list of ``(name, [sides])`` with sides from
    ``xmin,xmax,ymin,ymax,zmin,zmax``; every side must be used exactly once.
    With ``seed`` the cell numbering, the internal-face order and the face
    order inside each patch are permuted by ``numpy.random.default_rng(seed)``;
    owner < neighbour is kept for every internal face (faces are flipped where
    needed so their node order still points from owner to neighbour).

    ``skew`` > 0 moves every interior point by a seeded random offset of up
    to ``skew`` times the local spacing in each direction (points on the
    box's sides stay put), which makes the internal faces non-orthogonal
    (face normals no longer parallel to the owner-neighbour line) and the
    quads non-planar; keep it below about 0.25 so the cells stay convex.
    """
    if patches is None:
        patches = [(s, [s]) for s in SIDES]
    used = [s for _, ss in patches for s in ss]
    if sorted(used) != sorted(SIDES):
        raise ValueError("every side of the box must belong to exactly one patch")
    lx, ly, lz = lengths
    ox, oy, oz = origin
    xs = ox + lx * (np.arange(nx + 1, dtype=np.float64) / nx)
    ys = oy + ly * (np.arange(ny + 1, dtype=np.float64) / ny)
    zs = oz + lz * (np.arange(nz + 1, dtype=np.float64) / nz)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    points = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    if skew > 0.0:
        K, J, I = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
        inner = ((I > 0) & (I < nx) & (J > 0) & (J < ny) & (K > 0) & (K < nz)).ravel()
        rng = np.random.default_rng(skew_seed)
        off = rng.uniform(-skew, skew, size=(points.shape[0], 3)) * np.array([lx / nx, ly / ny, lz / nz])
        points = points + off * inner[:, None]

    def pid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    def cid(i, j, k):
        return i + nx * (j + ny * k)

    # ---- internal faces (node order points +axis: lower cell -> upper cell)
    quads, own, nei = [], [], []
    # x-faces at i = 1..nx-1
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(1, nx), indexing="ij")
    k, j, i = k.ravel(), j.ravel(), i.ravel()
    quads.append(np.stack([pid(i, j, k), pid(i, j + 1, k), pid(i, j + 1, k + 1), pid(i, j, k + 1)], 1))
    own.append(cid(i - 1, j, k)); nei.append(cid(i, j, k))
    # y-faces at j = 1..ny-1
    k, j, i = np.meshgrid(np.arange(nz), np.arange(1, ny), np.arange(nx), indexing="ij")
    k, j, i = k.ravel(), j.ravel(), i.ravel()
    quads.append(np.stack([pid(i, j, k), pid(i, j, k + 1), pid(i + 1, j, k + 1), pid(i + 1, j, k)], 1))
    own.append(cid(i, j - 1, k)); nei.append(cid(i, j, k))
    # z-faces at k = 1..nz-1
    k, j, i = np.meshgrid(np.arange(1, nz), np.arange(ny), np.arange(nx), indexing="ij")
    k, j, i = k.ravel(), j.ravel(), i.ravel()
    quads.append(np.stack([pid(i, j, k), pid(i + 1, j, k), pid(i + 1, j + 1, k), pid(i, j + 1, k)], 1))
    own.append(cid(i, j, k - 1)); nei.append(cid(i, j, k))
    iq = np.concatenate(quads).astype(np.int64)
    io = np.concatenate(own).astype(np.int64)
    ine = np.concatenate(nei).astype(np.int64)

    # ---- boundary faces per side (outward node order)
    side_faces = {}
    k, j = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
    k, j = k.ravel(), j.ravel()
    q = np.stack([pid(0, j, k), pid(0, j + 1, k), pid(0, j + 1, k + 1), pid(0, j, k + 1)], 1)
    side_faces["xmin"] = (q[:, ::-1], cid(0, j, k))
    q = np.stack([pid(nx, j, k), pid(nx, j + 1, k), pid(nx, j + 1, k + 1), pid(nx, j, k + 1)], 1)
    side_faces["xmax"] = (q, cid(nx - 1, j, k))
    k, i = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    k, i = k.ravel(), i.ravel()
    q = np.stack([pid(i, 0, k), pid(i, 0, k + 1), pid(i + 1, 0, k + 1), pid(i + 1, 0, k)], 1)
    side_faces["ymin"] = (q[:, ::-1], cid(i, 0, k))
    q = np.stack([pid(i, ny, k), pid(i, ny, k + 1), pid(i + 1, ny, k + 1), pid(i + 1, ny, k)], 1)
    side_faces["ymax"] = (q, cid(i, ny - 1, k))
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    j, i = j.ravel(), i.ravel()
    q = np.stack([pid(i, j, 0), pid(i + 1, j, 0), pid(i + 1, j + 1, 0), pid(i, j + 1, 0)], 1)
    side_faces["zmin"] = (q[:, ::-1], cid(i, j, 0))
    q = np.stack([pid(i, j, nz), pid(i + 1, j, nz), pid(i + 1, j + 1, nz), pid(i, j + 1, nz)], 1)
    side_faces["zmax"] = (q, cid(i, j, nz - 1))

    rng = np.random.default_rng(seed) if seed is not None else None
    ncell = nx * ny * nz
    cell_new = np.arange(ncell, dtype=np.int64)
    if rng is not None:
        cell_new = rng.permutation(ncell).astype(np.int64)
        order = rng.permutation(iq.shape[0])
        iq, io, ine = iq[order], io[order], ine[order]
    o2, n2 = cell_new[io], cell_new[ine]
    flip = o2 > n2
    iq = np.where(flip[:, None], iq[:, ::-1], iq)
    own_i = np.minimum(o2, n2)
    nei_i = np.maximum(o2, n2)

    bq, bo, names, sizes = [], [], [], []
    for name, ss in patches:
        q = np.concatenate([side_faces[s][0] for s in ss])
        c = np.concatenate([side_faces[s][1] for s in ss]).astype(np.int64)
        if rng is not None:
            order = rng.permutation(q.shape[0])
            q, c = q[order], c[order]
        bq.append(q)
        bo.append(cell_new[c])
        names.append(name)
        sizes.append(int(q.shape[0]))
    allq = np.concatenate([iq] + bq).astype(np.int32)
    owner = np.concatenate([own_i] + bo).astype(np.int32)
    nf = allq.shape[0]
    return PolyMesh(points=points, face_offsets=(4 * np.arange(nf + 1)).astype(np.int32),
                    face_nodes=allq.ravel().astype(np.int32), owner=owner,
                    neighbour=nei_i.astype(np.int32), patch_names=names, patch_sizes=sizes)


def cavity_polymesh(n: int = 80, seed: int | None = None, nx: int | None = None, lx: float = 1.0) -> PolyMesh:
    """Lid-driven cavity: [0, lx] x [0, 1] (unit square by default), an
    nx x n x 1 hex slab (nx = n by default) of thickness 1/n.

    Patches (in order): lid (y = 1), walls (x = 0, x = lx, y = 0),
    frontAndBack (z faces, Empty)."""
    nx = n if nx is None else nx
    return box_polymesh(nx, n, 1, lengths=(lx, 1.0, 1.0 / n),
                        patches=[("lid", ["ymax"]), ("walls", ["xmin", "xmax", "ymin"]),
                                 ("frontAndBack", ["zmin", "zmax"])], seed=seed)


def channel_polymesh(nx: int = 128, ny: int = 128, nz: int = 128, seed: int | None = 0,
                     length: float = 4.0) -> PolyMesh:
    """Steady channel: box [0,length]x[0,1]x[0,1] (length 4 by default);
    patches inlet (x = 0), outlet (x = length), walls (y and z sides);
    numbering permuted from ``seed``."""
    return box_polymesh(nx, ny, nz, lengths=(length, 1.0, 1.0),
                        patches=[("inlet", ["xmin"]), ("outlet", ["xmax"]),
                                 ("walls", ["ymin", "ymax", "zmin", "zmax"])], seed=seed)


def flatplate_polymesh(nx: int = 60, ny: int = 30, length: float = 0.5, height: float = 0.05,
                       seed: int | None = 0) -> PolyMesh:
    """2D flat plate (one cell deep): box [0,length]x[0,height]x[0,height/ny];
    patches inlet (x = 0), outlet (x = length), wall (y = 0), top (y =
    height), frontAndBack (the z sides, Empty); numbering permuted from
    ``seed``."""
    return box_polymesh(nx, ny, 1, lengths=(length, height, height / ny),
                        patches=[("inlet", ["xmin"]), ("outlet", ["xmax"]), ("wall", ["ymin"]), ("top", ["ymax"]),
                                 ("frontAndBack", ["zmin", "zmax"])], seed=seed)


def periodic_box_polymesh(n: int = 96, seed: int | None = None) -> PolyMesh:
    """Cube of side 2*pi with six patches xmin..zmax (periodic pairs)."""
    L = 2.0 * np.pi
    return box_polymesh(n, n, n, lengths=(L, L, L), patches=[(s, [s]) for s in SIDES], seed=seed)
