"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and the bench's
CPU-baseline leg as the checker.  The product never imports this module.
The oracle restates XCALibre.jl's CPU path in C++ (see orc_*.cpp for the
reference file:line each function follows).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_L = None


def build():
    env = dict(os.environ)
    env.pop("CXX", None)
    subprocess.run(["make", "-s", "-C", HERE], check=True, env=env)


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, i32, pd, pi = C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int)
        sig = {
            "orc_set_threads": (None, [i32]),
            "orc_get_threads": (i32, []),
            "orc_mesh_build": (vp, [i32, pd, i32, pi, pi, pi, i32, pi, i32, pi, C.c_char_p, i32]),
            "orc_mesh_from_desc": (vp, [vp]),
            "orc_mesh_free": (None, [vp]),
            "orc_mesh_sizes": (None, [vp, pi]),
            "orc_mesh_export": (None, [vp, pi, pi, pd, pd, pd, pd, pd, pd, pd, pd, pi, pi, pi, pi, pi, pi, pi]),
            "orc_construct_periodic": (i32, [vp, i32, i32, C.c_double, pi, pi, pd]),
            "orc_case_create": (vp, [vp, vp, C.c_char_p, i32]),
            "orc_case_free": (None, [vp]),
            "orc_case_nnz": (C.c_long, [vp, i32]),
            "orc_case_pattern": (None, [vp, i32, pi, pi]),
            "orc_case_get_system": (None, [vp, i32, i32, pd, pd]),
            "orc_case_set_field": (i32, [vp, i32, pd, C.c_long]),
            "orc_case_get_field": (i32, [vp, i32, pd, C.c_long]),
            "orc_case_mark_initialised": (i32, [vp]),
            "orc_simple_iterate": (i32, [vp, i32, pd, pi, pi]),
            "orc_piso_step": (i32, [vp, i32, pd, pd]),
            "orc_initial_calculations": (None, [vp]),
            "orc_discretise": (None, [vp, i32]),
            "orc_apply_bcs": (None, [vp, i32, i32]),
            "orc_relax": (None, [vp, i32]),
            "orc_set_reference": (None, [vp]),
            "orc_update_precond": (None, [vp, i32]),
            "orc_solve_system": (C.c_double, [vp, i32, i32, pi]),
            "orc_solve_equation": (None, [vp, i32, pd]),
            "orc_pressure_predictor": (None, [vp]),
            "orc_flux_divergence": (None, [vp]),
            "orc_prev_from_p": (None, [vp]),
            "orc_explicit_relaxation_p": (None, [vp, C.c_double]),
            "orc_grad_p": (None, [vp]),
            "orc_correct": (None, [vp]),
            "orc_turbulence": (None, [vp]),
            "orc_max_courant": (C.c_double, [vp]),
            "orc_canonical_sum": (C.c_double, [pd, C.c_long]),
            "orc_dilu": (None, [i32, pi, pi, pd, pd]),
            "orc_dilu_ldiv": (None, [i32, pi, pi, pd, pd, pd, pd]),
            "orc_jacobi_smooth": (None, [i32, pi, pi, pd, pd, pd, i32, C.c_double]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _L = L
    return _L


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def threads() -> int:
    return lib().orc_get_threads()


def canonical_sum(v) -> float:
    v = _d(v)
    return lib().orc_canonical_sum(_p(v, C.c_double), v.size)


class OracleMesh:
    def __init__(self, handle):
        self.h = handle

    @classmethod
    def from_polymesh(cls, pm):
        pts, fo, fn = _d(pm.points.ravel()), _i(pm.face_offsets), _i(pm.face_nodes)
        own, nei = _i(pm.owner), _i(pm.neighbour)
        ps = _i(pm.patch_sizes)
        err = C.create_string_buffer(256)
        h = lib().orc_mesh_build(pm.points.shape[0], _p(pts, C.c_double), pm.n_faces, _p(fo, C.c_int),
                                 _p(fn, C.c_int), _p(own, C.c_int), pm.n_internal_faces, _p(nei, C.c_int),
                                 len(pm.patch_sizes), _p(ps, C.c_int), err, 256)
        if not h:
            raise ValueError(err.value.decode())
        m = cls(h)
        m.patch_names = list(pm.patch_names)
        return m

    @classmethod
    def from_mesh3(cls, mesh3):
        # the product's Mesh3 arrays, as the Julia side would pass them
        import importlib
        abi = importlib.import_module("xcalibre_b200._abi")
        desc, keep = abi.mesh_desc(mesh3)
        h = lib().orc_mesh_from_desc(C.cast(C.pointer(desc), C.c_void_p))
        m = cls(h)
        m._keep = keep
        m.patch_names = list(mesh3.patch_names)
        return m

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_mesh_free(self.h)
            self.h = None

    def sizes(self):
        out = np.zeros(7, dtype=np.int32)
        lib().orc_mesh_sizes(self.h, _p(out, C.c_int))
        return dict(n_cells=int(out[0]), n_faces=int(out[1]), n_bfaces=int(out[2]), n_ifaces=int(out[3]),
                    n_patches=int(out[4]), n_cell_nodes=int(out[5]), n_points=int(out[6]))

    def export(self) -> dict:
        s = self.sizes()
        nC, nF, nB, nI, nP = s["n_cells"], s["n_faces"], s["n_bfaces"], s["n_ifaces"], s["n_patches"]
        a = dict(face_owner=np.zeros(nF, np.int32), face_neigh=np.zeros(nF, np.int32),
                 face_centre=np.zeros((nF, 3)), face_normal=np.zeros((nF, 3)), face_e=np.zeros((nF, 3)),
                 face_area=np.zeros(nF), face_delta=np.zeros(nF), face_weight=np.zeros(nF),
                 cell_centre=np.zeros((nC, 3)), cell_volume=np.zeros(nC),
                 cell_faces_offset=np.zeros(nC + 1, np.int32), cell_faces=np.zeros(2 * nI, np.int32),
                 cell_nsign=np.zeros(2 * nI, np.int32), cell_neighbours=np.zeros(2 * nI, np.int32),
                 boundary_cellsID=np.zeros(nB, np.int32), patch_start=np.zeros(nP, np.int32),
                 patch_count=np.zeros(nP, np.int32))
        order = ["face_owner", "face_neigh", "face_centre", "face_normal", "face_e", "face_area", "face_delta",
                 "face_weight", "cell_centre", "cell_volume", "cell_faces_offset", "cell_faces", "cell_nsign",
                 "cell_neighbours", "boundary_cellsID", "patch_start", "patch_count"]
        args = [_p(a[k], C.c_int if a[k].dtype == np.int32 else C.c_double) for k in order]
        lib().orc_mesh_export(self.h, *args)
        a.update(n_cells=nC, n_faces=nF, n_bfaces=nB)
        return a

    def construct_periodic(self, p1: int, p2: int, count: int, tol=1e-7):
        m1 = np.zeros(count, np.int32)
        m2 = np.zeros(count, np.int32)
        d = np.zeros(3)
        rc = lib().orc_construct_periodic(self.h, p1, p2, tol, _p(m1, C.c_int), _p(m2, C.c_int), _p(d, C.c_double))
        if rc != 0:
            raise ValueError(f"periodic matching failed ({rc})")
        return m1, m2, d


_FIELD_SHAPE = {0: (3, "cell"), 1: (1, "cell"), 2: (1, "face"), 3: (1, "face"), 4: (3, "cell"), 5: (9, "cell"),
                6: (1, "cell"), 7: (3, "cell"), 8: (1, "cell"), 9: (1, "cell"), 10: (1, "face"), 11: (3, "face"),
                12: (1, "face"), 13: (1, "face"), 14: (1, "cell"), 15: (1, "cell"), 16: (1, "cell"), 17: (1, "cell"),
                18: (1, "cell"), 19: (1, "cell"), 20: (1, "cell"), 21: (1, "cell"), 22: (1, "cell")}


class OracleCase:
    """Same methods as the product's Case, on the CPU oracle."""

    def __init__(self, omesh: OracleMesh, cfg):
        self.om = omesh
        s = omesh.sizes()
        self.nC, self.nF = s["n_cells"], s["n_faces"]
        err = C.create_string_buffer(256)
        self.h = lib().orc_case_create(omesh.h, C.cast(C.pointer(cfg), C.c_void_p), err, 256)
        if not self.h:
            raise ValueError(err.value.decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_case_free(self.h)
            self.h = None

    def _size(self, field):
        nc, kind = _FIELD_SHAPE[field]
        return nc, (self.nC if kind == "cell" else self.nF)

    def set_field(self, field, values):
        nc, per = self._size(field)
        a = _d(np.asarray(values, dtype=np.float64).reshape(nc * per))
        assert lib().orc_case_set_field(self.h, field, _p(a, C.c_double), a.size) == 0

    def mark_initialised(self):
        assert lib().orc_case_mark_initialised(self.h) == 0

    def get_field(self, field):
        nc, per = self._size(field)
        a = np.empty(nc * per)
        assert lib().orc_case_get_field(self.h, field, _p(a, C.c_double), a.size) == 0
        return a.reshape(nc, per) if nc > 1 else a

    def pattern(self, eqn):
        nnz = lib().orc_case_nnz(self.h, eqn)
        rp = np.empty(self.nC + 1, np.int32)
        cv = np.empty(nnz, np.int32)
        lib().orc_case_pattern(self.h, eqn, _p(rp, C.c_int), _p(cv, C.c_int))
        return rp, cv

    def system(self, eqn, component=0):
        nnz = lib().orc_case_nnz(self.h, eqn)
        nz = np.empty(nnz)
        b = np.empty(self.nC)
        lib().orc_case_get_system(self.h, eqn, component, _p(nz, C.c_double), _p(b, C.c_double))
        return nz, b

    def simple_iterate(self, n):
        res = np.zeros((max(n, 1), 4))
        done, conv = C.c_int(), C.c_int()
        lib().orc_simple_iterate(self.h, n, _p(res, C.c_double), C.byref(done), C.byref(conv))
        return res[: done.value], bool(conv.value)

    def piso_step(self, n):
        res = np.zeros((max(n, 1), 4))
        co = np.zeros(max(n, 1))
        lib().orc_piso_step(self.h, n, _p(res, C.c_double), _p(co, C.c_double))
        return res[:n], co[:n]

    def initial_calculations(self):
        lib().orc_initial_calculations(self.h)

    def discretise(self, eqn):
        lib().orc_discretise(self.h, eqn)

    def apply_boundary_conditions(self, eqn, comp=0):
        lib().orc_apply_bcs(self.h, eqn, comp)

    def implicit_relaxation_diagdom(self, comp):
        lib().orc_relax(self.h, comp)

    def set_reference(self):
        lib().orc_set_reference(self.h)

    def update_preconditioner(self, eqn):
        lib().orc_update_precond(self.h, eqn)

    def solve_system(self, eqn, comp=0):
        it = C.c_int()
        r = lib().orc_solve_system(self.h, eqn, comp, C.byref(it))
        return r, it.value

    def solve_equation(self, eqn):
        res = np.zeros(3)
        lib().orc_solve_equation(self.h, eqn, _p(res, C.c_double))
        return res if eqn == 0 else res[0]

    def pressure_predictor(self):
        lib().orc_pressure_predictor(self.h)

    def flux_divergence(self):
        lib().orc_flux_divergence(self.h)
        lib().orc_prev_from_p(self.h)

    def explicit_relaxation_p(self, alpha):
        lib().orc_explicit_relaxation_p(self.h, float(alpha))

    def grad_p(self):
        lib().orc_grad_p(self.h)

    def correct(self):
        lib().orc_correct(self.h)

    def turbulence(self):
        lib().orc_turbulence(self.h)

    def max_courant(self):
        return lib().orc_max_courant(self.h)


def dilu(rowptr, colval, nzval):
    n = len(rowptr) - 1
    D = np.zeros(n)
    rp, cv, nz = _i(rowptr), _i(colval), _d(nzval)
    lib().orc_dilu(n, _p(rp, C.c_int), _p(cv, C.c_int), _p(nz, C.c_double), _p(D, C.c_double))
    return D


def dilu_ldiv(rowptr, colval, nzval, D, b):
    n = len(rowptr) - 1
    x = np.zeros(n)
    rp, cv, nz, Dd, bb = _i(rowptr), _i(colval), _d(nzval), _d(D), _d(b)
    lib().orc_dilu_ldiv(n, _p(rp, C.c_int), _p(cv, C.c_int), _p(nz, C.c_double), _p(Dd, C.c_double),
                        _p(x, C.c_double), _p(bb, C.c_double))
    return x


def jacobi_smooth(rowptr, colval, nzval, b, x0, loops, omega):
    """apply_smoother!(JacobiSmoother(loops, omega)) on a CSR system from x0."""
    n = len(rowptr) - 1
    x = _d(x0).copy()
    rp, cv, nz, bb = _i(rowptr), _i(colval), _d(nzval), _d(b)
    lib().orc_jacobi_smooth(n, _p(rp, C.c_int), _p(cv, C.c_int), _p(nz, C.c_double), _p(bb, C.c_double),
                            _p(x, C.c_double), int(loops), float(omega))
    return x
