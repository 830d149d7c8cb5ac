"""LES{KEquation} (LES_KEquation.jl) on the CPU oracle.

A channel with a disturbed inflow runs PISO steps with the subgrid k
equation; after every step the oracle's fields satisfy the model's own
relations: nut = ck Delta sqrt(k) exactly (Delta = V^(1/3), the 3D
delta_scaling), k >= 0 (bound!), and the k-equation's cell sources, restated
here with numpy from the same grad U, nut and k (Pk = 2 nut grad U : dev(S),
the Si coefficients ce sqrt(k) / Delta and 2/3 tr grad U), are what the
oracle assembled."""
import numpy as np
import pytest


def _sources(G, nut, k, Delta, ce):
    """The k equation's cell sources (LES_KEquation.jl:164-168), the tensor
    products in the reference's order: G[a][b] = grad U component 3 a + b,
    the Frobenius product over column-major entries."""
    n = nut.size
    Pk, Dk, Dw = np.zeros(n), np.zeros(n), np.zeros(n)
    for i in range(n):
        g = G[:, i].reshape(3, 3)
        S = 0.5 * (g + g.T)
        third = (1.0 / 3.0) * ((S[0, 0] + S[1, 1]) + S[2, 2])
        dot = None
        for b in range(3):
            for a in range(3):
                pr = g[a, b] * (S[a, b] - third if a == b else S[a, b])
                dot = pr if dot is None else dot + pr
        Pk[i] = (2.0 * nut[i]) * dot
        Dk[i] = (ce * np.sqrt(k[i])) / Delta[i]
        Dw[i] = (2.0 / 3.0) * ((g[0, 0] + g[1, 1]) + g[2, 2])
    return Pk, Dk, Dw


def keq_oracle(x, orc, mesh, steps=3):
    model, config = x.cases.kequation_channel_case(mesh, steps=steps)
    cfg, keep = x.build_config(model, config)
    assert cfg.turbulence == x._abi.TURB_KEQUATION and cfg.keq_ck == 0.094 and cfg.keq_ce == 1.048
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    A = x._abi
    for f, v in (("FIELD_U", model.momentum.U), ("FIELD_P", model.momentum.p), ("FIELD_K", model.turbulence.k),
                 ("FIELD_NUT", model.turbulence.nut)):
        o.set_field(getattr(A, f), v)
    return o, model, config, (cfg, keep)


def test_kequation_relations(x, orc):
    mesh = x.build_mesh3(x.channel_polymesh(16, 8, 8, seed=3))
    o, model, config, keep = keq_oracle(x, orc, mesh)
    A = x._abi
    Delta = o.get_field(A.FIELD_DELTA)
    assert np.array_equal(Delta, np.power(mesh.cell_volume, 1.0 / 3.0))
    for step in range(3):
        nut0, k0 = o.get_field(A.FIELD_NUT).copy(), o.get_field(A.FIELD_K).copy()
        res, co = o.piso_step(1)
        assert np.all(np.isfinite(res)) and np.all(np.isfinite(co))
        k = o.get_field(A.FIELD_K)
        nut = o.get_field(A.FIELD_NUT)
        assert np.all(k >= 0.0)
        assert np.array_equal(nut, (0.094 * Delta) * np.sqrt(k))
        # the sources of this step's k equation, from its grad U, nut and k
        G = o.get_field(A.FIELD_GRADU).reshape(9, -1)
        Pk, Dk, Dw = _sources(G, nut0, k0, Delta, 1.048)
        assert np.array_equal(o.get_field(A.FIELD_PK), Pk)
        assert np.array_equal(o.get_field(A.FIELD_DK), Dk)
        assert np.array_equal(o.get_field(A.FIELD_DW), Dw)
    assert k.max() > 0.0 and nut.max() > 0.0


def test_kequation_periodic_oracle(x, orc):
    """On the periodic box the k equation runs with every field periodic:
    finite, k >= 0, nut = ck Delta sqrt(k)."""
    mesh = x.build_mesh3(x.periodic_box_polymesh(8, seed=2))
    U0 = x.cases.fourier_field(mesh, seed=2)
    model, config = x.cases.periodic_les_case(mesh, steps=3, U0=U0, model_kind=x.KEquation)
    cfg, keep = x.build_config(model, config)
    o = orc.OracleCase(orc.OracleMesh.from_mesh3(mesh), cfg)
    A = x._abi
    for f, v in (("FIELD_U", model.momentum.U), ("FIELD_P", model.momentum.p), ("FIELD_K", model.turbulence.k),
                 ("FIELD_NUT", model.turbulence.nut)):
        o.set_field(getattr(A, f), v)
    res, co = o.piso_step(3)
    assert np.all(np.isfinite(res)) and np.all(np.isfinite(co))
    k, nut = o.get_field(A.FIELD_K), o.get_field(A.FIELD_NUT)
    Delta = o.get_field(A.FIELD_DELTA)
    assert np.all(k >= 0.0) and k.max() > 0.0
    assert np.array_equal(nut, (0.094 * Delta) * np.sqrt(k))
