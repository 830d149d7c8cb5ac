"""GPU test of xcal_residual_noalloc, the entry point for callers that cannot
allocate device memory (graph capture, fixed budgets, caller-managed pools).

It must give the scaled residual xcal_solve_system reports for the same
system, on two calls in a row (the shared scratch array keeps the previous
call's contents).  The system is passed in the caller's original row order,
while the library sums rows in its own storage order, so the two agree to
rounding (the stated 1e-10), not bit for bit.  This file is collected last so
a failure here never hides other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10  # the FP64 parity tolerance of the other GPU tests


def test_noalloc_residual_matches_solve_system(x, ctx):
    import torch
    from importlib import import_module
    L = import_module("xcalibre_b200._lib").lib()
    A = x._abi
    mesh = x.build_mesh3(x.channel_polymesh(12, 6, 6, seed=5))
    model, config = x.cases.channel_case(mesh, iterations=1)
    cfg, keep = x.build_config(model, config)
    dm = x.DeviceMesh(ctx, mesh)
    case = x.Case(dm, cfg)
    rng = np.random.default_rng(1)
    case.set_field(A.FIELD_U, rng.standard_normal((3, mesh.n_cells)) * 0.1)
    case.initial_calculations()
    case.discretise(A.EQN_P)
    case.apply_boundary_conditions(A.EQN_P)
    case.update_preconditioner(A.EQN_P)
    res_existing, _ = case.solve_system(A.EQN_P)
    rp, cv = case.pattern(A.EQN_P)
    nz, b = case.system(A.EQN_P)
    p = case.get_field(A.FIELD_P)
    dev = torch.device("cuda", 0)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in
         dict(rp=rp, cv=cv, nz=nz, x=p, b=b).items()}
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    err = ctypes.create_string_buffer(256)
    results = []
    for _ in range(2):
        code = L.xcal_residual_noalloc(mesh.n_cells, t["rp"].data_ptr(), t["cv"].data_ptr(), t["nz"].data_ptr(),
                                       t["x"].data_ptr(), t["b"].data_ptr(), out.data_ptr(), None, err, 256)
        assert code == 0, err.value
        torch.cuda.synchronize()
        results.append(float(out.item()))
        out.fill_(-1.0)
    for r in results:
        assert abs(r - res_existing) <= TOL * abs(res_existing), (r, res_existing)
    # sizes beyond the fixed scratch are rejected with a message
    code = L.xcal_residual_noalloc(1 << 26, t["rp"].data_ptr(), t["cv"].data_ptr(), t["nz"].data_ptr(),
                                   t["x"].data_ptr(), t["b"].data_ptr(), out.data_ptr(), None, err, 256)
    assert code == A.XCAL_ERR_INVALID and b"33554432" in err.value
    case.close()
    dm.close()
