"""Mesh3 construction from a polyMesh (host side, once per mesh).

``build_mesh3`` calls the library's native importer (``xcal_foam_mesh_build``,
csrc/foam_import.cu), which restates XCALibre's ``FOAM3D_mesh`` pipeline
(src/FoamMesh/FoamMesh_*.jl, src/Mesh/Mesh_1_functions.jl:20-51) and needs no
GPU.  Indices are 0-based; faces 0..n_bfaces-1 are the boundary faces.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from .meshgen import PolyMesh


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
    polymesh: object = None      # the PolyMesh it was built from (nodes and faces, for the writers)
    dim: int = 3                 # 2: a Mesh2 (UNV2D_mesh), 3: a Mesh3
    cell_nodes: list | None = None  # 2D meshes read from UNV: each cell's nodes in element order (the 2D writer)

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
        return f"{self.dim}D Mesh with:\n-> {self.n_cells} cells\n-> {self.n_faces} faces\n-> {n_nodes} nodes"


def build_mesh3(pm: PolyMesh, device: int | None = None) -> Mesh3:
    """FOAM3D_mesh: polyMesh -> Mesh3 (Float64, 0-based) via the native
    importer; with ``device`` the geometry is computed on that GPU (the same
    result, for large meshes)."""
    from ._lib import lib
    keep = []

    def i32(a):
        a = np.ascontiguousarray(a, dtype=np.int32)
        keep.append(a)
        return _abi.ptr(a, C.c_int32)

    pts = np.ascontiguousarray(pm.points, dtype=np.float64)
    desc = _abi.PolyMeshDesc(n_points=pts.shape[0], points=_abi.ptr(pts, C.c_double), n_faces=pm.n_faces,
                             face_offsets=i32(pm.face_offsets), face_nodes=i32(pm.face_nodes), owner=i32(pm.owner),
                             n_internal_faces=pm.n_internal_faces, neighbour=i32(pm.neighbour),
                             n_patches=len(pm.patch_sizes), patch_sizes=i32(pm.patch_sizes))
    sizes = np.zeros(3, dtype=np.int32)
    if lib().xcal_foam_mesh_sizes(C.byref(desc), _abi.ptr(sizes, C.c_int32)) != 0:
        raise ValueError("invalid polyMesh")
    nC, nF, nB = (int(v) for v in sizes)
    nk = 2 * (nF - nB)
    m = Mesh3(n_cells=nC, n_faces=nF, n_bfaces=nB,
              face_owner=np.empty(nF, np.int32), face_neigh=np.empty(nF, np.int32),
              face_centre=np.empty((nF, 3)), face_normal=np.empty((nF, 3)), face_e=np.empty((nF, 3)),
              face_area=np.empty(nF), face_delta=np.empty(nF), face_weight=np.empty(nF),
              cell_centre=np.empty((nC, 3)), cell_volume=np.empty(nC),
              cell_faces_offset=np.empty(nC + 1, np.int32), cell_faces=np.empty(nk, np.int32),
              cell_nsign=np.empty(nk, np.int32), cell_neighbours=np.empty(nk, np.int32),
              boundary_cellsID=np.empty(nB, np.int32), patch_names=list(pm.patch_names),
              patch_start=np.empty(len(pm.patch_sizes), np.int32),
              patch_count=np.empty(len(pm.patch_sizes), np.int32), points=pts)
    out = _abi.MeshBuffers(**{f: _abi.ptr(getattr(m, f), C.c_int32 if getattr(m, f).dtype == np.int32 else C.c_double)
                              for f, _ in _abi.MeshBuffers._fields_})
    code = (lib().xcal_foam_mesh_build(C.byref(desc), C.byref(out)) if device is None else
            lib().xcal_foam_mesh_build_device(int(device), C.byref(desc), C.byref(out)))
    if code != 0:
        raise ValueError(f"invalid polyMesh (patch sizes, node or cell indices), or the device build failed ({code})")
    m.polymesh = pm
    return m
