"""ctypes mirror of the structs and constants in include/xcal_b200.h."""
from __future__ import annotations

import ctypes as C

import numpy as np

# status codes
XCAL_OK = 0
XCAL_ERR_INVALID = -1
XCAL_ERR_CUDA = -2
XCAL_ERR_OOM = -3
XCAL_ERR_NOT_CONVERGED = -4
XCAL_ERR_DIVERGED = -5
XCAL_ERR_TIMEOUT = -6
XCAL_ERR_UNSUPPORTED = -7
XCAL_ERR_BUSY = -8

# boundary conditions
BC_DIRICHLET = 1
BC_DIRICHLET_FUNCTION = 2
BC_WALL = 3
BC_ZEROGRADIENT = 4
BC_EXTRAPOLATED = 5
BC_EMPTY = 6
BC_SYMMETRY = 7
BC_NEUMANN = 8
BC_PERIODIC = 9
BC_PERIODIC_PARENT = 10
BC_OMEGA_WALL = 11
BC_K_WALL = 12
BC_NUT_WALL = 13

TIME_STEADY, TIME_EULER = 0, 1
DIV_LINEAR, DIV_UPWIND, DIV_LUST = 0, 1, 2
GRAD_GAUSS, GRAD_MIDPOINT = 0, 1
LIMITER_NONE, LIMITER_CELL, LIMITER_FACE, LIMITER_MFACE = 0, 1, 2, 3
SOLVER_CG, SOLVER_BICGSTAB = 0, 1
PRECOND_NONE, PRECOND_JACOBI, PRECOND_DILU = 0, 1, 2
TURB_LAMINAR, TURB_SMAGORINSKY, TURB_KOMEGA, TURB_KOMEGA_SST, TURB_KEQUATION, TURB_KOMEGA_LKE = 0, 1, 2, 3, 4, 5
PREC_FP64, PREC_MIXED = 0, 1
ALGO_SIMPLE, ALGO_PISO = 0, 1
EQN_U, EQN_P, EQN_K, EQN_OMEGA, EQN_WALLDIST, EQN_KL = 0, 1, 2, 3, 4, 5

FIELD_U, FIELD_P, FIELD_MDOTF, FIELD_NUEFF, FIELD_GRADP, FIELD_GRADU = 0, 1, 2, 3, 4, 5
FIELD_RD, FIELD_HV, FIELD_DIVHV, FIELD_NUT, FIELD_NUTF, FIELD_UF = 6, 7, 8, 9, 10, 11
FIELD_PF, FIELD_RDF, FIELD_DELTA, FIELD_K, FIELD_OMEGA, FIELD_WALLDIST = 12, 13, 14, 15, 16, 17
FIELD_PK, FIELD_DK, FIELD_DW, FIELD_KL, FIELD_GAMMA = 18, 19, 20, 21, 22

# (components, "cell"|"face") per field id
FIELD_SHAPE = {
    FIELD_U: (3, "cell"), FIELD_P: (1, "cell"), FIELD_MDOTF: (1, "face"), FIELD_NUEFF: (1, "face"),
    FIELD_GRADP: (3, "cell"), FIELD_GRADU: (9, "cell"), FIELD_RD: (1, "cell"), FIELD_HV: (3, "cell"),
    FIELD_DIVHV: (1, "cell"), FIELD_NUT: (1, "cell"), FIELD_NUTF: (1, "face"), FIELD_UF: (3, "face"),
    FIELD_PF: (1, "face"), FIELD_RDF: (1, "face"), FIELD_DELTA: (1, "cell"), FIELD_K: (1, "cell"),
    FIELD_OMEGA: (1, "cell"), FIELD_WALLDIST: (1, "cell"), FIELD_PK: (1, "cell"), FIELD_DK: (1, "cell"),
    FIELD_DW: (1, "cell"), FIELD_KL: (1, "cell"), FIELD_GAMMA: (1, "cell"),
}

_pi32 = C.POINTER(C.c_int32)
_pf64 = C.POINTER(C.c_double)


class MeshDesc(C.Structure):
    _fields_ = [
        ("n_cells", C.c_int32), ("n_faces", C.c_int32), ("n_bfaces", C.c_int32),
        ("face_owner", _pi32), ("face_neigh", _pi32),
        ("face_centre", _pf64), ("face_normal", _pf64), ("face_e", _pf64),
        ("face_area", _pf64), ("face_delta", _pf64), ("face_weight", _pf64),
        ("cell_centre", _pf64), ("cell_volume", _pf64),
        ("cell_faces_offset", _pi32), ("cell_faces", _pi32), ("cell_nsign", _pi32),
        ("cell_neighbours", _pi32), ("boundary_cellsID", _pi32),
        ("n_patches", C.c_int32), ("patch_start", _pi32), ("patch_count", _pi32), ("dim", C.c_int32),
    ]


class PolyMeshDesc(C.Structure):
    _fields_ = [
        ("n_points", C.c_int32), ("points", _pf64), ("n_faces", C.c_int32), ("face_offsets", _pi32),
        ("face_nodes", _pi32), ("owner", _pi32), ("n_internal_faces", C.c_int32), ("neighbour", _pi32),
        ("n_patches", C.c_int32), ("patch_sizes", _pi32),
    ]


class MeshBuffers(C.Structure):
    _fields_ = [
        ("face_owner", _pi32), ("face_neigh", _pi32), ("face_centre", _pf64), ("face_normal", _pf64),
        ("face_e", _pf64), ("face_area", _pf64), ("face_delta", _pf64), ("face_weight", _pf64),
        ("cell_centre", _pf64), ("cell_volume", _pf64), ("cell_faces_offset", _pi32), ("cell_faces", _pi32),
        ("cell_nsign", _pi32), ("cell_neighbours", _pi32), ("boundary_cellsID", _pi32), ("patch_start", _pi32),
        ("patch_count", _pi32),
    ]


class BCDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("patch", C.c_int32), ("value", C.c_double * 3),
        ("face_values", _pf64), ("face_map", _pi32), ("distance", C.c_double * 3),
        ("partner_patch", C.c_int32), ("wall", C.c_double * 5),
    ]


class SolverSetupDesc(C.Structure):
    _fields_ = [("solver", C.c_int32), ("precond", C.c_int32), ("convergence", C.c_double),
                ("relax", C.c_double), ("atol", C.c_double), ("rtol", C.c_double), ("itmax", C.c_int32),
                ("smoother_loops", C.c_int32), ("smoother_omega", C.c_double)]


class SchemesDesc(C.Structure):
    _fields_ = [("time", C.c_int32), ("divergence", C.c_int32), ("gradient", C.c_int32), ("limiter", C.c_int32),
                ("limiter_level", C.c_double)]


class ConfigDesc(C.Structure):
    _fields_ = [
        ("algorithm", C.c_int32), ("turbulence", C.c_int32), ("nu", C.c_double),
        ("smagorinsky_C", C.c_double), ("les_delta_distance", C.c_double), ("les_delta_power", C.c_double),
        ("U_schemes", SchemesDesc), ("p_schemes", SchemesDesc),
        ("U_solver", SolverSetupDesc), ("p_solver", SolverSetupDesc), ("iterations", C.c_int32),
        ("dt", C.c_double), ("has_pref", C.c_int32), ("pref", C.c_double), ("inner_loops", C.c_int32),
        ("ncorrectors", C.c_int32), ("precision", C.c_int32), ("inner_rtol", C.c_double), ("n_bc_U", C.c_int32), ("n_bc_p", C.c_int32), ("n_bc_nut", C.c_int32),
        ("bc_U", C.POINTER(BCDesc)), ("bc_p", C.POINTER(BCDesc)), ("bc_nut", C.POINTER(BCDesc)),
        ("kw_beta_star", C.c_double), ("kw_alpha1", C.c_double), ("kw_beta1", C.c_double),
        ("kw_sigma_k", C.c_double), ("kw_sigma_omega", C.c_double),
        ("k_schemes", SchemesDesc), ("omega_schemes", SchemesDesc),
        ("k_solver", SolverSetupDesc), ("omega_solver", SolverSetupDesc),
        ("n_bc_k", C.c_int32), ("n_bc_omega", C.c_int32),
        ("bc_k", C.POINTER(BCDesc)), ("bc_omega", C.POINTER(BCDesc)),
        ("sst_beta2", C.c_double), ("sst_sigma_k2", C.c_double), ("sst_sigma_omega2", C.c_double),
        ("y_schemes", SchemesDesc), ("y_solver", SolverSetupDesc), ("n_bc_y", C.c_int32),
        ("bc_y", C.POINTER(BCDesc)), ("keq_ck", C.c_double), ("keq_ce", C.c_double),
        ("lke_Tu", C.c_double), ("kl_schemes", SchemesDesc), ("kl_solver", SolverSetupDesc), ("n_bc_kl", C.c_int32),
        ("bc_kl", C.POINTER(BCDesc)),
    ]


OP_TIME, OP_DIVERGENCE, OP_LAPLACIAN, OP_SI = 0, 1, 2, 3


class TermDesc(C.Structure):
    _fields_ = [("op", C.c_int32), ("scheme", C.c_int32), ("sign", C.c_double), ("flux", _pf64),
                ("value", C.c_double)]


class SourceDesc(C.Structure):
    _fields_ = [("sign", C.c_double), ("field", _pf64), ("value", C.c_double)]


def ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def mesh_desc(mesh) -> tuple[MeshDesc, list]:
    """Build an xcal_mesh_desc from a Mesh3; returns (desc, keepalive list)."""
    keep = []

    def i32(a):
        a = np.ascontiguousarray(a, dtype=np.int32)
        keep.append(a)
        return ptr(a, C.c_int32)

    def f64(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return ptr(a, C.c_double)

    d = MeshDesc(
        n_cells=mesh.n_cells, n_faces=mesh.n_faces, n_bfaces=mesh.n_bfaces,
        face_owner=i32(mesh.face_owner), face_neigh=i32(mesh.face_neigh),
        face_centre=f64(mesh.face_centre), face_normal=f64(mesh.face_normal), face_e=f64(mesh.face_e),
        face_area=f64(mesh.face_area), face_delta=f64(mesh.face_delta), face_weight=f64(mesh.face_weight),
        cell_centre=f64(mesh.cell_centre), cell_volume=f64(mesh.cell_volume),
        cell_faces_offset=i32(mesh.cell_faces_offset), cell_faces=i32(mesh.cell_faces),
        cell_nsign=i32(mesh.cell_nsign), cell_neighbours=i32(mesh.cell_neighbours),
        boundary_cellsID=i32(mesh.boundary_cellsID), n_patches=len(mesh.patch_start),
        patch_start=i32(mesh.patch_start), patch_count=i32(mesh.patch_count), dim=int(getattr(mesh, "dim", 3)))
    return d, keep
