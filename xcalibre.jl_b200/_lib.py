"""ctypes binding of libxcal_b200.so (the C ABI in include/xcal_b200.h).

The library is required: there is no CPU fallback.  Loading fails loudly when
the shared object has not been built.
"""
from __future__ import annotations

import ctypes as C
import os

from . import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxcal_b200.so")

_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int32)
_pi64 = C.POINTER(C.c_int64)

# name -> (restype, argtypes); every symbol declared in include/xcal_b200.h
SIGNATURES = {
    "xcal_ctx_create": (_i32, [_i32, C.POINTER(_vp)]),
    "xcal_ctx_destroy": (_i32, [_vp]),
    "xcal_last_error": (C.c_char_p, [_vp]),
    "xcal_version": (C.c_char_p, []),
    "xcal_foam_mesh_sizes": (_i32, [C.POINTER(_abi.PolyMeshDesc), _pi]),
    "xcal_foam_mesh_build": (_i32, [C.POINTER(_abi.PolyMeshDesc), C.POINTER(_abi.MeshBuffers)]),
    "xcal_foam_mesh_build_device": (_i32, [_i32, C.POINTER(_abi.PolyMeshDesc), C.POINTER(_abi.MeshBuffers)]),
    "xcal_mesh_upload": (_i32, [_vp, C.POINTER(_abi.MeshDesc), C.POINTER(_vp)]),
    "xcal_mesh_destroy": (_i32, [_vp]),
    "xcal_case_create": (_i32, [_vp, _vp, C.POINTER(_abi.ConfigDesc), C.POINTER(_vp)]),
    "xcal_case_destroy": (_i32, [_vp]),
    "xcal_case_nnz": (_i32, [_vp, _i32, _pi64]),
    "xcal_case_csr_pattern": (_i32, [_vp, _i32, _pi, _pi]),
    "xcal_case_get_system": (_i32, [_vp, _i32, _i32, _pd, _pd]),
    "xcal_case_set_field": (_i32, [_vp, _i32, _pd, _i64]),
    "xcal_case_get_field": (_i32, [_vp, _i32, _pd, _i64]),
    "xcal_case_set_bc_values": (_i32, [_vp, _i32, _i32, _pd, _i64]),
    "xcal_simple_iterate": (_i32, [_vp, _i32, _pd, _pi, _pi]),
    "xcal_piso_step": (_i32, [_vp, _i32, _pd, _pd, _pi]),
    "xcal_initial_calculations": (_i32, [_vp]),
    "xcal_discretise": (_i32, [_vp, _i32]),
    "xcal_apply_boundary_conditions": (_i32, [_vp, _i32, _i32]),
    "xcal_implicit_relaxation_diagdom": (_i32, [_vp, _i32]),
    "xcal_set_reference": (_i32, [_vp]),
    "xcal_update_preconditioner": (_i32, [_vp, _i32]),
    "xcal_solve_system": (_i32, [_vp, _i32, _i32, _pd, _pi]),
    "xcal_solve_equation": (_i32, [_vp, _i32, _pd]),
    "xcal_pressure_predictor": (_i32, [_vp]),
    "xcal_flux_divergence": (_i32, [_vp]),
    "xcal_explicit_relaxation_p": (_i32, [_vp, C.c_double]),
    "xcal_grad_p": (_i32, [_vp]),
    "xcal_correct": (_i32, [_vp]),
    "xcal_turbulence": (_i32, [_vp]),
    "xcal_max_courant": (_i32, [_vp, _pd]),
    "xcal_get_timings": (_i32, [_vp, _pd, _i32]),
    "xcal_get_launch_count": (_i32, [_vp, _pi64]),
    "xcal_case_stream": (_i32, [_vp, C.POINTER(_vp)]),
    "xcal_case_set_profiling": (_i32, [_vp, _i32]),
    "xcal_case_set_graph_mode": (_i32, [_vp, _i32]),
    "xcal_case_set_persistent": (_i32, [_vp, _i32]),
    "xcal_case_mark_initialised": (_i32, [_vp]),
    "xcal_case_tuning": (_i32, [_vp, _pi]),
    "xcal_case_set_dilu_mode": (_i32, [_vp, _i32]),
    "xcal_case_set_inner_cg": (_i32, [_vp, _i32]),
    "xcal_abi_layout": (_i32, [_i32, C.POINTER(C.c_int64), _i32]),
    "xcal_case_solve_report": (_i32, [_vp, _pi, _pi, _pi64]),
    "xcal_check_bounded_wait": (_i32, [_vp, _i64, _pi, _pi, _pi]),
    "xcal_det_math": (_i32, [_i32, _pd, _pd, _i64]),
    "xcal_equation_create": (_i32, [_vp, _i32, C.POINTER(_abi.TermDesc), _i32, C.POINTER(_abi.SourceDesc), _i32,
                                    C.POINTER(_abi.BCDesc), C.POINTER(_vp)]),
    "xcal_equation_destroy": (_i32, [_vp]),
    "xcal_equation_discretise": (_i32, [_vp, _pd, C.c_double]),
    "xcal_equation_apply_bcs": (_i32, [_vp, _pd]),
    "xcal_equation_nnz": (_i32, [_vp, _pi64]),
    "xcal_equation_get_system": (_i32, [_vp, _pi, _pi, _pd, _pd]),
    "xcal_equation_solve": (_i32, [_vp, C.POINTER(_abi.SolverSetupDesc), _pd, _pd, _pi]),
    "xcal_case_get_profile": (_i32, [_vp, _i32, _pd, _pi64]),
    "xcal_residual_noalloc": (_i32, [_i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_char_p, _i32]),
    "xcal_footprint_estimate": (_i32, [_i64, _i64, _i64, _i32, _i32, _i32, _pi64]),
    "xcal_case_footprint": (_i32, [_vp, _pi64, _pi64]),
    "xcal_batch_create": (_i32, [_vp, _i32, _i64, C.POINTER(_vp)]),
    "xcal_batch_destroy": (_i32, [_vp]),
    "xcal_batch_add": (_i32, [_vp, _vp, _i64]),
    "xcal_batch_remove": (_i32, [_vp, _vp]),
    "xcal_batch_info": (_i32, [_vp, _pi, _pi64, _pi64]),
    "xcal_batch_case_index": (_i32, [_vp, _vp, _pi]),
    "xcal_batch_timings": (_i32, [_vp, _pd]),
    "xcal_batch_simple_iterate": (_i32, [_vp, _pd, _pi]),
}

_LIB = None


def lib():
    """Load libxcal_b200.so (raises if it is missing)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run __graft_entry__.build() "
                               "or python xcalibre.jl_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


class XcalError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"xcal error {code}: {msg}")
        self.code = code


def check(code: int, ctx) -> None:
    if code != _abi.XCAL_OK:
        msg = lib().xcal_last_error(ctx).decode() if ctx else ""
        raise XcalError(code, msg)
