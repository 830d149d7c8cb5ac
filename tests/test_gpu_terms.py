"""Scalar equations from the operator DSL through the term-list ABI
(xcal_equation_*), on the GPU:

* unit_test_laplace.jl:112-130, (-Laplacian{Linear}(1, T) == -Source(0)) ->
  ScalarEquation(T, BCs), written with the DSL: its A and b are the golden
  ones;
* SIMPLE's pressure equation, (-Laplacian{Linear}(rDf, p) == -Source(divHv))
  -> ScalarEquation(p, BCs.p) (Solvers_1_SIMPLE.jl:76-78), from the case's
  own rDf and divHv: the driver's assembled system bit for bit (the driver's
  is pinned to the oracle by the parity tests);
* a transport equation with every operator (Time{Euler}, Divergence with
  Linear / Upwind / LUST, Laplacian, Si; two sources) and every scalar
  boundary type, on a skewed mesh: equal to a plain-Python restatement of
  discretise! and apply_boundary_conditions! in the reference's order
  (Discretise_2_generated_distretisation.jl:125-167, Discretise_1_schemes.jl,
  boundary_conditions/*.jl), to 1e-13 relative;
* the DSL's sign rule (ModelFramework_1_operations.jl:3-19);
* solve_system! on a Dirichlet Poisson problem: CG + Jacobi and BiCGSTAB +
  DILU reach the direct solution of the exported system.
"""
import numpy as np
import pytest

from test_oracle_golden import _laplace_mesh, laplace_check

pytestmark = pytest.mark.gpu


def _dsl(x):
    from importlib import import_module
    return import_module(x.__name__ + ".dsl")


def _laplace_case(x, ctx, m):
    model = x.Physics(time=x.Steady(), fluid=x.Fluid(x.Incompressible, nu=1.0), turbulence=x.RANS(x.Laminar),
                      energy=x.Energy(x.Isothermal), domain=m)
    BCs = x.assign(region=m, U=[x.Zerogradient(n) for n in m.patch_names[:4]] + [x.Empty("frontAndBack")],
                   p=[x.Zerogradient(n) for n in m.patch_names[:4]] + [x.Empty("frontAndBack")])
    solvers = {s: x.SolverSetup(solver=x.Cg(), preconditioner=x.Jacobi(), convergence=1e-8, relax=0.8)
               for s in ("U", "p")}
    config = x.Configuration(solvers=solvers, schemes={"U": x.Schemes(), "p": x.Schemes()},
                             runtime=x.Runtime(iterations=1, write_interval=1, time_step=1.0),
                             hardware=x.Hardware(backend=x.B200Backend()), boundaries=BCs)
    cfg, keep = x.build_config(model, config)
    dm = x.DeviceMesh(ctx, m)
    return x.Case(dm, cfg), (cfg, keep, dm)


def test_sign_rule(x):
    D = _dsl(x)
    T = np.zeros(4)
    a, b, c = D.Laplacian[x.Linear](1.0, T), D.Si(2.0, T), D.Time[x.Euler](T)
    m = (a - b + c == D.Source(1.0) - D.Source(2.0))
    assert [t.sign for t in m.terms] == [1.0, -1.0, 1.0]
    assert [s.sign for s in m.sources] == [1.0, -1.0]
    m2 = (-a == -D.Source(0.0))
    assert [t.sign for t in m2.terms] == [-1.0] and [s.sign for s in m2.sources] == [-1.0]
    # `-` sets the sign, it does not flip it (Base.:-(a, b) sets b.sign = -1)
    m3 = (a - (-b)[0] == D.Source(0.0))
    assert [t.sign for t in m3.terms] == [1.0, -1.0]


def test_laplace_golden_from_terms(x, ctx):
    D = _dsl(x)
    m = _laplace_mesh(x)
    case, keep = _laplace_case(x, ctx, m)
    T = np.zeros(m.n_cells)
    bcs = [x.Dirichlet("left_wall", 50.0), x.Zerogradient("right_wall"), x.Dirichlet("bottom_wall", 10.0),
           x.Zerogradient("upper_wall"), x.Empty("frontAndBack")]
    eqn = (-D.Laplacian[x.Linear](1.0, T) == -D.Source(0.0)) >> D.ScalarEquation(T, bcs)
    E = D.Equation(case, eqn)
    E.discretise()
    E.apply_boundary_conditions(T)
    rp, cv, nz, b = E.system()
    laplace_check(m, nz, rp, cv, b)
    E.close()


def test_pressure_equation_from_terms_matches_driver(x, ctx):
    D = _dsl(x)
    A = x._abi
    mesh = x.build_mesh3(x.channel_polymesh(14, 8, 7, seed=5))
    model, config = x.cases.channel_case(mesh, iterations=2)
    cfg, keep = x.build_config(model, config)
    dm = x.DeviceMesh(ctx, mesh)
    case = x.Case(dm, cfg)
    rng = np.random.default_rng(2)
    case.set_field(A.FIELD_U, rng.standard_normal((3, mesh.n_cells)) * 0.1)
    case.set_field(A.FIELD_P, rng.standard_normal(mesh.n_cells) * 0.01)
    case.initial_calculations()
    case.discretise(A.EQN_U)
    for d in range(3):
        case.apply_boundary_conditions(A.EQN_U, d)
    case.pressure_predictor()
    case.flux_divergence()
    case.discretise(A.EQN_P)
    case.apply_boundary_conditions(A.EQN_P)
    nz_drv, b_drv = case.system(A.EQN_P)
    rp_drv, cv_drv = case.pattern(A.EQN_P)
    rDf, divHv, p = case.get_field(A.FIELD_RDF), case.get_field(A.FIELD_DIVHV), case.get_field(A.FIELD_P)
    eqn = (-D.Laplacian[x.Linear](rDf, p) == -D.Source(divHv)) >> D.ScalarEquation(p, config.boundaries["p"])
    E = D.Equation(case, eqn)
    E.discretise()
    E.apply_boundary_conditions(p)
    rp, cv, nz, b = E.system()
    assert np.array_equal(rp, rp_drv) and np.array_equal(cv, cv_drv)
    assert np.array_equal(nz, nz_drv) and np.array_equal(b, b_drv)
    E.close()


def _restate(mesh, terms, sources, bcs_by_patch, prev, dt, phi):
    """discretise! + apply_boundary_conditions! of a scalar equation, in
    plain Python, the reference's term and face order (original numbering)."""
    n = mesh.n_cells
    A = {}
    b = np.zeros(n)
    nrm, ee = mesh.face_normal, mesh.face_e
    for i in range(n):
        ac_sum = 0.0
        for k in range(mesh.cell_faces_offset[i], mesh.cell_faces_offset[i + 1]):
            f, ns, j = mesh.cell_faces[k], float(mesh.cell_nsign[k]), mesh.cell_neighbours[k]
            AC = AN = 0.0
            for t in terms:
                fl = (t["flux"][f] if np.ndim(t["flux"]) else t["flux"]) if t["op"] in ("lap", "div") else 0.0
                if t["op"] == "lap":
                    Sf = [ns * mesh.face_area[f] * nrm[f, c] for c in range(3)]
                    e = [ns * ee[f, c] for c in range(3)]
                    r = (Sf[0] * Sf[0] + Sf[1] * Sf[1] + Sf[2] * Sf[2]) / (Sf[0] * e[0] + Sf[1] * e[1] + Sf[2] * e[2])
                    Ef = np.sqrt((r * e[0]) ** 2 + (r * e[1]) ** 2 + (r * e[2]) ** 2)
                    ap = (t["sign"] * (fl * Ef)) / mesh.face_delta[f]
                    ac, an = -ap, ap
                elif t["op"] == "div":
                    ap = t["sign"] * (fl * ns)
                    w = mesh.face_weight[f]
                    if t["scheme"] == "linear":
                        w = 0.5 + ns * (w - 0.5)
                        ac, an = ap * w, ap * (1.0 - w)
                    elif t["scheme"] == "upwind":
                        ac, an = max(ap, 0.0), -max(-ap, 0.0)
                    else:
                        if ns < 0:
                            w = 1.0 - w
                        ac = 0.75 * (ap * w) + 0.25 * max(ap, 0.0)
                        an = 0.75 * (ap * (1.0 - w)) + 0.25 * (-max(-ap, 0.0))
                else:
                    ac = an = 0.0
                AC += ac
                AN += an
            ac_sum += AC
            A[(i, j)] = AN
        V = mesh.cell_volume[i]
        acs = bs = 0.0
        for t in terms:
            fl = (t["flux"][i] if np.ndim(t["flux"]) else t["flux"]) if t["op"] in ("time", "si") else 0.0
            if t["op"] == "time":
                vr = (fl * V) / dt
                acs += vr
                bs += prev[i] * vr
            elif t["op"] == "si":
                acs += (t["sign"] * fl) * V
        A[(i, i)] = ac_sum + acs
        b2 = 0.0
        for s in sources:
            b2 += (s["sign"] * (s["field"][i] if np.ndim(s["field"]) else s["field"])) * V
        b[i] = b2 + bs
    for f in range(mesh.n_bfaces):
        c = mesh.face_owner[f]
        kind, val = bcs_by_patch[f]
        ap = bp = 0.0
        for t in terms:
            fl = (t["flux"][f] if np.ndim(t["flux"]) else t["flux"]) if t["op"] in ("lap", "div") else 0.0
            a = q = 0.0
            if t["op"] == "lap":
                if kind == "dirichlet":
                    a = t["sign"] * (-((fl * mesh.face_area[f]) / mesh.face_delta[f]))
                    q = a * val
                elif kind == "extrapolated":
                    a = t["sign"] * (((-fl) * mesh.face_area[f]) / mesh.face_delta[f])
                    q = a * phi[c]
                elif kind == "neumann":
                    q = (fl * mesh.face_area[f]) * val
            elif t["op"] == "div":
                if kind == "dirichlet":
                    q = (t["sign"] * (-fl)) * val
                elif kind == "neumann":
                    a = t["sign"] * fl
                    q = ((-val) * a) * mesh.face_delta[f]
                elif kind != "empty":
                    a = t["sign"] * fl
            ap += a
            bp += q
        A[(c, c)] += ap
        b[c] += bp
    return A, b


@pytest.mark.parametrize("div", ["linear", "upwind", "lust"])
def test_transport_equation_matches_restatement(x, ctx, div):
    D = _dsl(x)
    mesh = x.build_mesh3(x.box_polymesh(7, 5, 4, seed=3, skew=0.15))
    case, keep = _laplace_case_generic(x, ctx, mesh)
    rng = np.random.default_rng(7)
    nC, nF = mesh.n_cells, mesh.n_faces
    phi = rng.uniform(0.5, 1.5, nC)
    prev = rng.uniform(0.5, 1.5, nC)
    mdot = rng.standard_normal(nF) * 0.3
    gam = rng.uniform(0.1, 2.0, nF)
    si = rng.uniform(0.0, 3.0, nC)
    s1, s2 = rng.standard_normal(nC), rng.standard_normal(nC)
    dt = 0.013
    scheme = {"linear": x.Linear, "upwind": x.Upwind, "lust": x.LUST}[div]
    bcs = [x.Dirichlet("xmin", 1.5), x.Neumann("xmax", 0.3), x.Extrapolated("ymin"), x.Zerogradient("ymax"),
           x.Wall("zmin"), x.Symmetry("zmax")]
    eqn = (D.Time[x.Euler](phi) + D.Divergence[scheme](mdot, phi) - D.Laplacian[x.Linear](gam, phi)
           + D.Si(si, phi) == D.Source(s1) - D.Source(s2)) >> D.ScalarEquation(phi, bcs)
    E = D.Equation(case, eqn)
    E.discretise(prev, dt)
    E.apply_boundary_conditions(phi)
    rp, cv, nz, b = E.system()
    terms = [dict(op="time", flux=1.0, sign=1.0), dict(op="div", flux=mdot, sign=1.0, scheme=div),
             dict(op="lap", flux=gam, sign=-1.0), dict(op="si", flux=si, sign=1.0)]
    sources = [dict(field=s1, sign=1.0), dict(field=s2, sign=-1.0)]
    kinds = {"xmin": ("dirichlet", 1.5), "xmax": ("neumann", 0.3), "ymin": ("extrapolated", 0.0),
             "ymax": ("zerogradient", 0.0), "zmin": ("wall", 0.0), "zmax": ("symmetry", 0.0)}
    bc_f = {}
    for name, (k, v) in kinds.items():
        for f in mesh.patch_range(name):
            bc_f[f] = (k, v)
    Ar, br = _restate(mesh, terms, sources, bc_f, prev, dt, phi)
    dense = np.zeros((nC, nC))
    for i in range(nC):
        for e in range(rp[i], rp[i + 1]):
            dense[i, cv[e]] = nz[e]
    ref = np.zeros((nC, nC))
    for (i, j), v in Ar.items():
        ref[i, j] = v
    assert np.allclose(dense, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
    assert np.allclose(b, br, rtol=1e-13, atol=1e-13 * np.abs(br).max())
    E.close()


def _laplace_case_generic(x, ctx, m):
    """A case on mesh m whose own equations are not used (it carries the
    mesh, stream and Krylov workspace the term-list equation runs on)."""
    model = x.Physics(time=x.Steady(), fluid=x.Fluid(x.Incompressible, nu=1.0), turbulence=x.RANS(x.Laminar),
                      energy=x.Energy(x.Isothermal), domain=m)
    BCs = x.assign(region=m, U=[x.Zerogradient(n) for n in m.patch_names],
                   p=[x.Zerogradient(n) for n in m.patch_names])
    solvers = {s: x.SolverSetup(solver=x.Cg(), preconditioner=x.Jacobi(), convergence=1e-8, relax=0.8)
               for s in ("U", "p")}
    config = x.Configuration(solvers=solvers, schemes={"U": x.Schemes(), "p": x.Schemes()},
                             runtime=x.Runtime(iterations=1, write_interval=1, time_step=1.0),
                             hardware=x.Hardware(backend=x.B200Backend()), boundaries=BCs)
    cfg, keep = x.build_config(model, config)
    dm = x.DeviceMesh(ctx, m)
    return x.Case(dm, cfg), (cfg, keep, dm)


@pytest.mark.parametrize("solver,pre", [("cg", "jacobi"), ("bicgstab", "dilu")])
def test_poisson_solve_from_terms(x, ctx, solver, pre):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    D = _dsl(x)
    mesh = x.build_mesh3(x.box_polymesh(12, 10, 8, seed=4))
    case, keep = _laplace_case_generic(x, ctx, mesh)
    rng = np.random.default_rng(3)
    T = np.zeros(mesh.n_cells)
    src = rng.uniform(0.0, 1.0, mesh.n_cells)
    bcs = [x.Dirichlet("xmin", 1.0), x.Dirichlet("xmax", 0.0), x.Zerogradient("ymin"), x.Zerogradient("ymax"),
           x.Zerogradient("zmin"), x.Zerogradient("zmax")]
    eqn = (-D.Laplacian[x.Linear](1.0, T) == D.Source(src)) >> D.ScalarEquation(T, bcs)
    E = D.Equation(case, eqn)
    E.discretise()
    E.apply_boundary_conditions(T)
    rp, cv, nz, b = E.system()
    Asp = sp.csr_matrix((nz, cv, rp), shape=(mesh.n_cells, mesh.n_cells))
    exact = spl.spsolve(Asp.tocsc(), b)
    setup = x.SolverSetup(solver=x.Cg() if solver == "cg" else x.Bicgstab(),
                          preconditioner=x.Jacobi() if pre == "jacobi" else x.DILU(),
                          convergence=1e-10, relax=1.0, rtol=1e-12, atol=1e-14, itmax=5000)
    sol, res, its = E.solve(setup, T)
    assert its > 0 and res < 1e-10, (res, its)
    assert np.linalg.norm(sol - exact) / np.linalg.norm(exact) < 1e-8
    E.close()
