"""RANS{KOmegaLKE} (RANS_kOmegaLKE.jl) on the CPU oracle.

* its cell loops against a numpy restatement written from the reference's
  formulas (with numpy's exp and power): after one SIMPLE iteration of the
  flat plate of examples/2D_flatplate_LKE_ERCOFTAC.jl, the intermittency
  gamma (:309-323), the k equation's source and Si coefficient (:401-420;
  the production term `sum(g .* 2*S_dev)` is Julia's left-to-right
  (g .* 2) * S_dev, a matrix product), omega's Si coefficient (:381) and
  nut (:436-460) from the observable fields before and after the call;
* a few hundred iterations stay finite with gamma in [0, 1] and kl, k,
  omega bounded below by eps (bound!, RANS_functions.jl:2-41);
* the configuration mapping (Tu, kl's BCs / schemes / solver, the wall BCs
  of the wall distance)."""
import numpy as np
import pytest

KL_FIELDS = ("FIELD_U", "FIELD_P", "FIELD_K", "FIELD_OMEGA", "FIELD_KL", "FIELD_NUT")


def flatplate(x, nx=24, ny=12, seed=0):
    return x.build_mesh3(x.flatplate_polymesh(nx, ny, seed=seed))


def set_lke_fields(x, c, model):
    t = model.turbulence
    for f, v in (("FIELD_U", model.momentum.U), ("FIELD_P", model.momentum.p), ("FIELD_K", t.k),
                 ("FIELD_OMEGA", t.omega), ("FIELD_KL", t.kl), ("FIELD_NUT", t.nut)):
        c.set_field(getattr(x._abi, f), v)


def lke_cells(gradU, U, y, nu, eta, kl0, k0, w0, kl1, k1, w1):
    """The cell loops of turbulence!(::KOmegaLKEModel) as the reference
    writes them, vectorised over cells."""
    n = U.shape[1]
    G = gradU.reshape(3, 3, n).transpose(2, 0, 1)  # [cell, a, b] = d u_a / d x_b
    divU = np.trace(G, axis1=1, axis2=2)
    Sd = 0.5 * (G + G.transpose(0, 2, 1)) - (divU / 3.0)[:, None, None] * np.eye(3)
    S2 = 2.0 * np.sum(Sd ** 2, axis=(1, 2))
    Om = np.sqrt(2.0 * np.sum((0.5 * (G - G.transpose(0, 2, 1))) ** 2, axis=(1, 2)))
    PkA = np.sum((G * 2.0) @ Sd, axis=(1, 2))
    normU = np.sqrt(np.sum(U * U, axis=0))
    ReL = np.maximum(normU, np.sqrt(np.finfo(float).eps)) * y / nu

    def reu(kl):
        return np.sqrt(np.sqrt(2.0 * nu ** 2 * kl / y ** 2)) * y / nu

    den = np.maximum(S2, (normU / y) ** 2)
    nutL1 = eta * kl0 * np.sqrt(S2) * reu(kl0) ** -1.30 * ReL ** 0.5 / den
    ReLt = np.minimum(kl0 / np.maximum(np.minimum(nu, nutL1), 1e-15) / np.maximum(Om, 1e-15), 5000.0)
    gam = np.minimum(ReLt ** 2, 76500.0) / 76500.0
    sw1, sk0 = np.maximum(w1, 1e-15), np.maximum(k0, 1e-15)
    fv = 1.0 - np.exp(-np.sqrt(sk0 / (max(nu, 1e-15) * sw1)) / 0.43)
    Pk = np.minimum(fv * (sk0 / sw1) * PkA * gam, 20.0 * 0.09 * sk0 * w1) - (2.0 / 3.0) * divU * k0
    Dk = 0.09 * gam * w1
    Dw = 0.0708 * w0
    PkL = np.sqrt(S2) * eta * kl1 * reu(kl1) ** -1.30 * ReL ** 0.5
    sk1 = np.maximum(k1, 1e-15)
    fSS = np.exp(-(1.45 * nu * Om / sk1) ** 2)
    nut = fSS * (sk1 / np.maximum(w1, 1e-15)) + PkL / den
    return dict(gam=gam, Pk=Pk, Dk=Dk, Dw=Dw, nut=nut)


def close(a, b, rtol=1e-9):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) <= rtol * max(np.max(np.abs(b)), 1e-300)


def test_lke_config_mapping(x):
    mesh = flatplate(x)
    model, config = x.cases.lke_flatplate_case(mesh, 5, Tu=0.03)
    cfg, keep = x.build_config(model, config)
    A = x._abi
    assert cfg.turbulence == A.TURB_KOMEGA_LKE and cfg.lke_Tu == 0.03
    assert cfg.n_bc_kl == 5 and cfg.bc_kl[0].type == A.BC_DIRICHLET and cfg.bc_kl[0].value[0] == 0.0115
    assert cfg.kl_schemes.divergence == A.DIV_LUST and cfg.kl_solver.relax == 0.3
    # wall_distance!: Dirichlet 0 on the walls, Empty, Extrapolated elsewhere
    assert [cfg.bc_y[i].type for i in range(cfg.n_bc_y)] == [A.BC_EXTRAPOLATED, A.BC_EXTRAPOLATED, A.BC_DIRICHLET,
                                                              A.BC_EXTRAPOLATED, A.BC_EMPTY]
    with pytest.raises(ValueError):
        x.build_config(x.api.Physics(time=x.api.Steady(), fluid=model.fluid, turbulence=x.api.RANS(x.api.KOmegaLKE),
                                     energy=model.energy, domain=mesh), config)


def test_lke_cell_loops_restated(x, orc):
    mesh = flatplate(x)
    model, config = x.cases.lke_flatplate_case(mesh, 1)
    cfg, keep = x.build_config(model, config)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    set_lke_fields(x, o, model)
    A, t = x._abi, model.turbulence
    o.simple_iterate(1)
    g = {f: o.get_field(getattr(A, f)) for f in ("FIELD_GRADU", "FIELD_U", "FIELD_WALLDIST", "FIELD_KL", "FIELD_K",
                                                   "FIELD_OMEGA", "FIELD_GAMMA", "FIELD_PK", "FIELD_DK", "FIELD_DW",
                                                   "FIELD_NUT")}
    Tu = 0.01
    eta = 0.02974 * np.tanh(59.79 * Tu ** 1.191 + 1.65e-13)
    ref = lke_cells(g["FIELD_GRADU"], g["FIELD_U"], g["FIELD_WALLDIST"], 1.48e-5, eta, t.kl, t.k, t.omega,
                    g["FIELD_KL"], g["FIELD_K"], g["FIELD_OMEGA"])
    assert np.all((g["FIELD_GAMMA"] > 0.0) & (g["FIELD_GAMMA"] <= 1.0))
    for name, f in (("gam", "FIELD_GAMMA"), ("Pk", "FIELD_PK"), ("Dk", "FIELD_DK"), ("Dw", "FIELD_DW"),
                    ("nut", "FIELD_NUT")):
        assert close(g[f], ref[name]), name


def test_lke_flatplate_bounded(x, orc):
    mesh = flatplate(x, 20, 10)
    model, config = x.cases.lke_flatplate_case(mesh, 200)
    cfg, keep = x.build_config(model, config)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    set_lke_fields(x, o, model)
    res, _ = o.simple_iterate(200)
    assert np.all(np.isfinite(res))
    eps = np.finfo(float).eps
    for f in ("FIELD_K", "FIELD_OMEGA", "FIELD_KL"):
        v = o.get_field(getattr(x._abi, f))
        assert np.all(np.isfinite(v)) and v.min() >= eps, f
    gam = o.get_field(x._abi.FIELD_GAMMA)
    assert np.all((gam >= 0.0) & (gam <= 1.0))
    nut = o.get_field(x._abi.FIELD_NUT)
    assert np.all(np.isfinite(nut)) and nut.min() >= 0.0
