"""CellBased gradient limiter (Calculate_0_gradient_cell_limiter.jl:68-108;
applied after every grad p, Solvers_1_SIMPLE.jl:154/193/206, and after grad U
in the turbulence update, RANS_laminar.jl:77) on the CPU oracle, skewed
channel: with level 1 every gradient-extrapolated face value stays inside the
cell's neighbour range (Barth-Jespersen bound); level 0 gives the unlimited
run bit for bit; the API checks level and refuses unknown limiters.

FaceBased (Calculate_0_gradient_face_limiter.jl): after limiting, every
cell's gradient, extrapolated to each of its internal faces, stays inside
the bounds min/max(F_owner, F_neighbour) widened by their difference (the
scalar form, checked for p); the vector form leaves every cell's gradient a
non-negative multiple (at most 1) of the unlimited one computed from the same
fields."""
import numpy as np
import pytest

from test_nonorth_oracle import skewed_channel


def _run(x, orc, mesh, p_lim=None, U_lim=None, iters=4, ncorr=0):
    model, config = x.cases.channel_case(mesh, iterations=iters)
    config.schemes["p"].limiter = p_lim
    config.schemes["U"].limiter = U_lim
    cfg, keep = x.build_config(model, config, ncorrectors=ncorr)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    o.set_field(x._abi.FIELD_U, model.momentum.U)
    o.set_field(x._abi.FIELD_P, model.momentum.p)
    res, _ = o.simple_iterate(iters)
    return res, {f: o.get_field(f) for f in (x._abi.FIELD_U, x._abi.FIELD_P, x._abi.FIELD_GRADP,
                                               x._abi.FIELD_GRADU)}


def _check_bound(mesh, F, g):
    """F_P + (fc - cc).g within [min, max] of F over P and its neighbours, for
    every internal face of every cell (rounding allowance 1e-9 of the range)."""
    off, cf, nb = mesh.cell_faces_offset, mesh.cell_faces, mesh.cell_neighbours
    fc, cc = np.asarray(mesh.face_centre), np.asarray(mesh.cell_centre)
    cells = np.repeat(np.arange(mesh.n_cells), np.diff(off))
    d = fc[cf] - cc[cells]
    ext = F[cells] + np.einsum("kd,dk->k", d, g[:, cells])
    hi = np.maximum.reduceat(np.maximum(F[nb], F[cells]), off[:-1])
    lo = np.minimum.reduceat(np.minimum(F[nb], F[cells]), off[:-1])
    tol = 1e-9 * (np.ptp(F) + 1e-300)
    assert np.all(ext <= hi[cells] + tol) and np.all(ext >= lo[cells] - tol)


def test_limiter_bounds_and_acts(x, orc):
    mesh = skewed_channel(x)
    res0, f0 = _run(x, orc, mesh)
    res1, f1 = _run(x, orc, mesh, p_lim=x.api.CellBased(1.0), U_lim=x.api.CellBased(1.0))
    assert np.all(np.isfinite(res1))
    assert not np.array_equal(f0[x._abi.FIELD_GRADP], f1[x._abi.FIELD_GRADP])
    assert not np.array_equal(f0[x._abi.FIELD_GRADU], f1[x._abi.FIELD_GRADU])
    _check_bound(mesh, f1[x._abi.FIELD_P], f1[x._abi.FIELD_GRADP])
    U, gU = f1[x._abi.FIELD_U], f1[x._abi.FIELD_GRADU]
    for a in range(3):
        _check_bound(mesh, U[a], gU[3 * a:3 * a + 3])
    # the unlimited gradients break the bound somewhere (the limiter had work)
    with pytest.raises(AssertionError):
        _check_bound(mesh, f0[x._abi.FIELD_P], f0[x._abi.FIELD_GRADP])


def test_limiter_level_zero_is_identity(x, orc):
    mesh = skewed_channel(x, seed=5)
    res0, f0 = _run(x, orc, mesh, ncorr=1)
    res1, f1 = _run(x, orc, mesh, p_lim=x.api.CellBased(0.0), U_lim=x.api.CellBased(0.0), ncorr=1)
    assert np.array_equal(res0, res1)
    for k in f0:
        assert np.array_equal(f0[k], f1[k]), k


def test_limiter_api(x):
    with pytest.raises(ValueError):
        x.api.CellBased(1.5)
    with pytest.raises(ValueError):
        x.api.CellBased(-0.1)
    mesh = skewed_channel(x, n=(4, 3, 3))
    model, config = x.cases.channel_case(mesh, iterations=1)
    config.schemes["p"].limiter = object()
    with pytest.raises(NotImplementedError):
        x.build_config(model, config)
    config.schemes["p"].limiter = x.api.MFaceBased(mesh)
    cfg, keep = x.build_config(model, config)
    assert cfg.p_schemes.limiter == x._abi.LIMITER_MFACE
    config.schemes["p"].limiter = x.api.FaceBased(mesh)
    cfg, keep = x.build_config(model, config)
    assert cfg.p_schemes.limiter == x._abi.LIMITER_FACE


def _check_face_bound(mesh, F, g):
    """F_P + (fc - cc).g within [min - d, max + d] of the face's two cells'
    values, d = max - min, for every internal face of every cell."""
    off, cf, nb = mesh.cell_faces_offset, mesh.cell_faces, mesh.cell_neighbours
    fc, cc = np.asarray(mesh.face_centre), np.asarray(mesh.cell_centre)
    cells = np.repeat(np.arange(mesh.n_cells), np.diff(off))
    d = fc[cf] - cc[cells]
    ext = F[cells] + np.einsum("kd,dk->k", d, g[:, cells])
    hi = np.maximum(F[nb], F[cells])
    lo = np.minimum(F[nb], F[cells])
    w = hi - lo
    tol = 1e-9 * (np.ptp(F) + 1e-300)
    assert np.all(ext <= hi + w + tol) and np.all(ext >= lo - w - tol)


def test_face_limiter_bounds(x, orc):
    mesh = skewed_channel(x, seed=7)
    res0, f0 = _run(x, orc, mesh)
    res1, f1 = _run(x, orc, mesh, p_lim=x.api.FaceBased(mesh), U_lim=x.api.FaceBased(mesh))
    assert np.all(np.isfinite(res1))
    assert not np.array_equal(f0[x._abi.FIELD_GRADP], f1[x._abi.FIELD_GRADP])
    _check_face_bound(mesh, f1[x._abi.FIELD_P], f1[x._abi.FIELD_GRADP])
    with pytest.raises(AssertionError):
        _check_face_bound(mesh, f0[x._abi.FIELD_P], f0[x._abi.FIELD_GRADP])


def test_face_limiter_vector_scales(x, orc):
    """The vector form scales each cell's whole gradient tensor by one
    factor in [0, 1]: one oracle iteration with and without it from the same
    state gives gradients in that ratio, cell by cell."""
    mesh = skewed_channel(x, seed=8)
    res, f = _run(x, orc, mesh, iters=1)
    _, fl = _run(x, orc, mesh, U_lim=x.api.FaceBased(mesh), iters=1)
    G0, G1 = f[x._abi.FIELD_GRADU], fl[x._abi.FIELD_GRADU]
    n0 = np.linalg.norm(G0, axis=0)
    ok = n0 > 0
    ratio = np.linalg.norm(G1, axis=0)[ok] / n0[ok]
    assert np.all(ratio <= 1.0 + 1e-12) and np.all(ratio >= 0.0) and np.any(ratio < 1.0)
    # parallel: G1 = ratio * G0 per cell
    assert np.allclose(G1[:, ok], G0[:, ok] * ratio, rtol=1e-12, atol=0.0)


def _mface_loop(mesh, F, g):
    """limit_gradient!(::MFaceBased) (Calculate_0_gradient_mface_limiter.jl)
    as its kernel reads, run on one thread: internal faces in id order, each
    correcting its owner's then its neighbour's gradient.  F: [n] (g [3, n])
    or [3, n] (g [9, n], rows of grad U); vector bounds are Base's min / max
    of two vectors, chosen whole by the lexicographic order."""
    g = np.array(g, dtype=np.float64)
    fc, cc = np.asarray(mesh.face_centre), np.asarray(mesh.cell_centre)
    own, nei = np.asarray(mesh.face_owner), np.asarray(mesh.face_neigh)
    vec = F.ndim == 2
    for f in range(mesh.n_bfaces, mesh.n_faces):
        o, n = own[f], nei[f]
        if vec:
            F1, F2 = F[:, o], F[:, n]
            lt = tuple(F2) < tuple(F1)
            mx, mn = (F1, F2) if lt else (F2, F1)
        else:
            mx, mn = max(F[o], F[n]), min(F[o], F[n])
        for c in (o, n):
            d = fc[f] - cc[c]
            d2 = d @ d
            rows = range(3) if vec else [None]
            for a in rows:
                sl = slice(3 * a, 3 * a + 3) if vec else slice(0, 3)
                hi = (mx[a] - F[a, c]) if vec else (mx - F[c])
                lo = (mn[a] - F[a, c]) if vec else (mn - F[c])
                fval = g[sl, c] @ d
                if fval > hi:
                    g[sl, c] = g[sl, c] + d * (hi - fval) / d2
                elif fval < lo:
                    g[sl, c] = g[sl, c] + d * (lo - fval) / d2
    return g


def _green_gauss(mesh, pf):
    """sum over a cell's faces of phi_f S_f / V (Calculate_0_gradient.jl)"""
    S = np.asarray(mesh.face_normal) * np.asarray(mesh.face_area)[:, None]
    own, nei = np.asarray(mesh.face_owner), np.asarray(mesh.face_neigh)
    g = np.zeros((3, mesh.n_cells))
    nB = mesh.n_bfaces
    np.add.at(g.T, own, pf[:, None] * S)
    np.add.at(g.T, nei[nB:], -(pf[nB:, None] * S[nB:]))
    return g / np.asarray(mesh.cell_volume)


def test_mface_limiter_restated(x, orc):
    """The oracle's per-cell form equals the reference's face loop on one
    thread: p's limited gradient against the loop applied to the Green-Gauss
    gradient of the same face values; grad U against the loop applied to the
    unlimited grad U of the same U (a laminar iteration's U does not depend
    on its U limiter)."""
    mesh = skewed_channel(x, seed=9)
    model, config = x.cases.channel_case(mesh, iterations=1)
    config.schemes["p"].limiter = x.api.MFaceBased(mesh)
    cfg, keep = x.build_config(model, config)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    o.set_field(x._abi.FIELD_U, model.momentum.U)
    o.set_field(x._abi.FIELD_P, model.momentum.p)
    o.simple_iterate(1)
    P, pf, gp = (o.get_field(f) for f in (x._abi.FIELD_P, x._abi.FIELD_PF, x._abi.FIELD_GRADP))
    ref = _mface_loop(mesh, P, _green_gauss(mesh, pf))
    assert np.max(np.abs(gp - ref)) <= 1e-9 * np.max(np.abs(ref))
    assert not np.allclose(ref, _green_gauss(mesh, pf))  # the limiter acted
    _, f0 = _run(x, orc, mesh, iters=1)
    _, f1 = _run(x, orc, mesh, U_lim=x.api.MFaceBased(mesh), iters=1)
    assert np.array_equal(f0[x._abi.FIELD_U], f1[x._abi.FIELD_U])
    refU = _mface_loop(mesh, f0[x._abi.FIELD_U], f0[x._abi.FIELD_GRADU])
    G1 = f1[x._abi.FIELD_GRADU]
    assert np.max(np.abs(G1 - refU)) <= 1e-9 * np.max(np.abs(refU))
    assert not np.array_equal(G1, f0[x._abi.FIELD_GRADU])
