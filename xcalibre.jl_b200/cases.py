"""The benchmark workloads, written with the reference-style API.

* cavity_case        -- 2D lid-driven cavity (80x80x1, Re = 100), SIMPLE,
                        Upwind, CG+Jacobi (p), BiCGSTAB+DILU (U), relax 0.7/0.3
                        (after examples/2D_cavity.jl:30-83 with the stated solvers)
* channel_case       -- 3D steady laminar channel 4x1x1, parabolic inlet
                        (peak 1 m/s), zeroGradient outlet, no-slip walls,
                        nu = 1e-3, LUST, SIMPLE
* periodic_les_case  -- periodic cube, PISO + Smagorinsky (Cs = 0.17),
                        Euler, Linear divergence, nu = 1e-4; initial field
                        from fourier_field (seeded, k^4 exp(-2 (k/4)^2));
                        or the subgrid k equation (LES{KEquation})
* kequation_channel_case -- the channel with LES{KEquation}, PISO
* lke_flatplate_case -- steady RANS{KOmegaLKE} flat plate (Tu = 0.01, U =
                        5.4 m/s, nu = 1.48e-5), after
                        examples/2D_flatplate_LKE_ERCOFTAC.jl:16-151
"""
from __future__ import annotations

import numpy as np

from . import api as A
from .foam import Mesh3


def _solvers(U_pre=A.DILU, p_pre=A.Jacobi, relax_U=0.7, relax_p=0.3, conv=1e-7, rtol_U=0.1, rtol_p=0.1):
    return {
        "U": A.SolverSetup(solver=A.Bicgstab(), preconditioner=U_pre(), convergence=conv, relax=relax_U,
                           rtol=rtol_U),
        "p": A.SolverSetup(solver=A.Cg(), preconditioner=p_pre(), convergence=conv, relax=relax_p, rtol=rtol_p),
    }


def cavity_case(mesh: Mesh3, iterations: int = 1000, precision: str = "fp64", device: int = 0, nu: float = 0.01):
    # nu = 0.01: Re = 100 on the unit square with lid speed 1
    model = A.Physics(time=A.Steady(), fluid=A.Fluid(A.Incompressible, nu=nu), turbulence=A.RANS(A.Laminar),
                      energy=A.Energy(A.Isothermal), domain=mesh)
    BCs = A.assign(
        region=mesh,
        U=[A.Wall("lid", [1.0, 0.0, 0.0]), A.Wall("walls", [0.0, 0.0, 0.0]), A.Empty("frontAndBack")],
        p=[A.Wall("lid"), A.Wall("walls"), A.Empty("frontAndBack")],
    )
    schemes = {"U": A.Schemes(divergence=A.Upwind), "p": A.Schemes()}
    config = A.Configuration(solvers=_solvers(), schemes=schemes,
                             runtime=A.Runtime(iterations=iterations, write_interval=-1, time_step=1.0),
                             hardware=A.Hardware(backend=A.B200Backend(device=device, precision=precision)),
                             boundaries=BCs)
    A.initialise_(model.momentum.U, [0.0, 0.0, 0.0])
    A.initialise_(model.momentum.p, 0.0)
    return model, config


def parabolic_inlet(coords, time, index):
    """U_x = 16 y(1-y) z(1-z): peak 1 m/s at the centre of the unit section."""
    y, z = coords[1], coords[2]
    return [16.0 * y * (1.0 - y) * z * (1.0 - z), 0.0, 0.0]


def channel_case(mesh: Mesh3, iterations: int = 500, precision: str = "fp64", device: int = 0,
                 convergence: float = 1e-6, nu: float = 1e-3):
    model = A.Physics(time=A.Steady(), fluid=A.Fluid(A.Incompressible, nu=nu), turbulence=A.RANS(A.Laminar),
                      energy=A.Energy(A.Isothermal), domain=mesh)
    BCs = A.assign(
        region=mesh,
        U=[A.DirichletFunction("inlet", parabolic_inlet), A.Zerogradient("outlet"), A.Wall("walls", [0.0, 0.0, 0.0])],
        p=[A.Zerogradient("inlet"), A.Dirichlet("outlet", 0.0), A.Wall("walls")],
    )
    schemes = {"U": A.Schemes(divergence=A.LUST), "p": A.Schemes()}
    config = A.Configuration(solvers=_solvers(conv=convergence), schemes=schemes,
                             runtime=A.Runtime(iterations=iterations, write_interval=-1, time_step=1.0),
                             hardware=A.Hardware(backend=A.B200Backend(device=device, precision=precision)),
                             boundaries=BCs)
    A.initialise_(model.momentum.U, [0.0, 0.0, 0.0])
    A.initialise_(model.momentum.p, 0.0)
    return model, config


def kequation_channel_case(mesh: Mesh3, steps: int = 20, precision: str = "fp64", device: int = 0,
                           nu: float = 1e-4, dt: float = 2e-3, k_in: float = 1e-3, ck: float = 0.094,
                           ce: float = 1.048, seed: int = 0):
    """LES{KEquation} on the channel (PISO, Euler, Linear divergence): the
    parabolic inlet with inflow k = k_in, walls with k = 0 and nut = 0, a
    seeded disturbance of U (5% of the inlet peak) and k = k_in inside."""
    model = A.Physics(time=A.Transient(), fluid=A.Fluid(A.Incompressible, nu=nu),
                      turbulence=A.LES(A.KEquation, ck=ck, ce=ce), energy=A.Energy(A.Isothermal), domain=mesh)
    BCs = A.assign(
        region=mesh,
        U=[A.DirichletFunction("inlet", parabolic_inlet), A.Zerogradient("outlet"), A.Wall("walls", [0.0, 0.0, 0.0])],
        p=[A.Zerogradient("inlet"), A.Dirichlet("outlet", 0.0), A.Wall("walls")],
        k=[A.Dirichlet("inlet", k_in), A.Zerogradient("outlet"), A.Dirichlet("walls", 0.0)],
        nut=[A.Zerogradient("inlet"), A.Zerogradient("outlet"), A.Dirichlet("walls", 0.0)],
    )
    lin = A.Schemes(time=A.Euler, divergence=A.Linear)
    s = _solvers(relax_U=1.0, relax_p=1.0, rtol_U=0.1, rtol_p=0.01)
    s["k"] = A.SolverSetup(solver=A.Bicgstab(), preconditioner=A.Jacobi(), convergence=1e-7, relax=1.0, rtol=1e-3)
    config = A.Configuration(solvers=s, schemes={"U": lin, "p": A.Schemes(), "k": lin},
                             runtime=A.Runtime(iterations=steps, write_interval=-1, time_step=dt),
                             hardware=A.Hardware(backend=A.B200Backend(device=device, precision=precision)),
                             boundaries=BCs)
    rng = np.random.default_rng(seed)
    U = np.zeros((3, mesh.n_cells))
    U[0] = 1.0
    U += 0.05 * rng.standard_normal(U.shape)
    model.momentum.U[:] = U
    A.initialise_(model.momentum.p, 0.0)
    A.initialise_(model.turbulence.k, k_in)
    A.initialise_(model.turbulence.nut, 0.0)
    return model, config


def lke_flatplate_case(mesh: Mesh3, iterations: int = 1000, precision: str = "fp64", device: int = 0,
                       precond=A.Jacobi, Tu: float = 0.01):
    """RANS{KOmegaLKE} on the flat plate (patches inlet, outlet, wall, top,
    frontAndBack): inflow 5.4 m/s with k = 0.0575, kl = 0.0115, omega = 275;
    OmegaWallFunction on the wall, Extrapolated on the top; LUST divergence;
    the solvers, relaxation and initial fields of the reference example."""
    velocity, nu = [5.4, 0.0, 0.0], 1.48e-5
    k_in, kl_in, w_in = 0.0575, 0.0115, 275.0
    model = A.Physics(time=A.Steady(), fluid=A.Fluid(A.Incompressible, nu=nu),
                      turbulence=A.RANS(A.KOmegaLKE, Tu=Tu, walls=["wall"]), energy=A.Energy(A.Isothermal),
                      domain=mesh)
    fb = A.Empty("frontAndBack")
    BCs = A.assign(
        region=mesh,
        U=[A.Dirichlet("inlet", velocity), A.Zerogradient("outlet"), A.Wall("wall", [0.0, 0.0, 0.0]),
           A.Extrapolated("top"), fb],
        p=[A.Zerogradient("inlet"), A.Dirichlet("outlet", 0.0), A.Wall("wall"), A.Extrapolated("top"), fb],
        k=[A.Dirichlet("inlet", k_in), A.Zerogradient("outlet"), A.Dirichlet("wall", 0.0), A.Extrapolated("top"), fb],
        kl=[A.Dirichlet("inlet", kl_in), A.Zerogradient("outlet"), A.Dirichlet("wall", 0.0), A.Extrapolated("top"),
            fb],
        omega=[A.Dirichlet("inlet", w_in), A.Zerogradient("outlet"), A.OmegaWallFunction("wall"),
               A.Extrapolated("top"), fb],
        nut=[A.Dirichlet("inlet", k_in / w_in), A.Extrapolated("outlet"), A.Dirichlet("wall", 0.0),
             A.Extrapolated("top"), fb],
    )
    lust = A.Schemes(divergence=A.LUST)

    def ss(solver, relax, conv=1e-8, rtol=1e-2):
        return A.SolverSetup(solver=solver(), preconditioner=precond(), convergence=conv, relax=relax, rtol=rtol)

    solvers = {"U": ss(A.Bicgstab, 0.7), "p": ss(A.Cg, 0.2, rtol=1e-3),
               "y": A.SolverSetup(solver=A.Cg(), preconditioner=A.Jacobi(), convergence=1e-7, relax=0.9, rtol=1e-3),
               "kl": ss(A.Bicgstab, 0.3), "k": ss(A.Bicgstab, 0.3), "omega": ss(A.Bicgstab, 0.3)}
    schemes = {"U": lust, "p": A.Schemes(divergence=A.LUST), "k": lust, "y": A.Schemes(), "kl": lust, "omega": lust}
    config = A.Configuration(solvers=solvers, schemes=schemes,
                             runtime=A.Runtime(iterations=iterations, write_interval=-1, time_step=1.0),
                             hardware=A.Hardware(backend=A.B200Backend(device=device, precision=precision)),
                             boundaries=BCs)
    A.initialise_(model.momentum.U, velocity)
    A.initialise_(model.momentum.p, 0.0)
    A.initialise_(model.turbulence.kl, kl_in)
    A.initialise_(model.turbulence.k, k_in)
    A.initialise_(model.turbulence.omega, w_in)
    A.initialise_(model.turbulence.nut, k_in / w_in)
    return model, config


def taylor_green(mesh: Mesh3, rms: float = 1.0) -> np.ndarray:
    """Divergence-free periodic field on [0, 2pi]^3 (deterministic)."""
    x, y, z = mesh.cell_centre[:, 0], mesh.cell_centre[:, 1], mesh.cell_centre[:, 2]
    U = np.stack([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z), np.zeros_like(x)])
    cur = np.sqrt(np.mean(np.sum(U * U, axis=0)))
    return U * (rms / cur)


def fourier_field(mesh: Mesh3, seed: int = 0, k0: float = 4.0, rms: float = 1.0,
                  L: float = 2.0 * np.pi) -> np.ndarray:
    """Seeded random divergence-free velocity on the periodic cube [0, L]^3.

    Spectral method: random complex Fourier coefficients on the n^3 integer
    wavenumber grid with amplitude sqrt(E(k) / (4 pi k^2)), E(k) = k^4
    exp(-2 (k/k0)^2), projected onto k . u = 0 (u - k (k.u)/|k|^2); the real
    part of the inverse FFT is sampled at the cell centres (the box mesh is a
    uniform lattice, cells may be numbered in any order) and scaled to the
    requested rms of |U|.  Shape (3, n_cells)."""
    nc = mesh.n_cells
    n = int(round(nc ** (1.0 / 3.0)))
    if n ** 3 != nc:
        raise ValueError("fourier_field needs an n^3 box mesh")
    rng = np.random.default_rng(seed)
    k1 = np.fft.fftfreq(n, d=1.0 / n) * (2.0 * np.pi / L)
    kx, ky, kz = np.meshgrid(k1, k1, k1, indexing="ij")
    kk = kx * kx + ky * ky + kz * kz
    kmag = np.sqrt(kk)
    with np.errstate(divide="ignore", invalid="ignore"):
        E = kmag ** 4 * np.exp(-2.0 * (kmag / k0) ** 2)
        amp = np.where(kmag > 0, np.sqrt(E / (4.0 * np.pi * np.where(kk > 0, kk, 1.0))), 0.0)
    u = [amp * (rng.standard_normal(kk.shape) + 1j * rng.standard_normal(kk.shape)) for _ in range(3)]
    kdu = kx * u[0] + ky * u[1] + kz * u[2]
    inv = np.where(kk > 0, 1.0 / np.where(kk > 0, kk, 1.0), 0.0)
    u = [u[0] - kx * kdu * inv, u[1] - ky * kdu * inv, u[2] - kz * kdu * inv]
    grid = np.stack([np.real(np.fft.ifftn(c)) for c in u])
    h = L / n
    idx = np.clip(np.floor(mesh.cell_centre / h).astype(np.int64), 0, n - 1)
    U = grid[:, idx[:, 0], idx[:, 1], idx[:, 2]]
    cur = np.sqrt(np.mean(np.sum(U * U, axis=0)))
    return U * (rms / cur)


def periodic_les_case(mesh: Mesh3, steps: int = 200, dt: float | None = None, precision: str = "fp64",
                      device: int = 0, U0: np.ndarray | None = None, model_kind=None, k0: float = 1e-3):
    """The periodic LES box: Smagorinsky (C = 0.17) by default, or
    model_kind=A.KEquation (the subgrid k equation, k = k0 initially, every
    field periodic)."""
    pairs = [A.construct_periodic(mesh, None, a, b) for a, b in (("xmin", "xmax"), ("ymin", "ymax"), ("zmin", "zmax"))]
    per = [bc for pair in pairs for bc in pair]
    keq = model_kind is A.KEquation
    turb = A.LES(A.KEquation) if keq else A.LES(A.Smagorinsky, C=0.17)
    model = A.Physics(time=A.Transient(), fluid=A.Fluid(A.Incompressible, nu=1e-4), turbulence=turb,
                      energy=A.Energy(A.Isothermal), domain=mesh)
    BCs = A.assign(region=mesh, U=per, p=per, nut=per, **({"k": per} if keq else {}))
    schemes = {"U": A.Schemes(time=A.Euler, divergence=A.Linear), "p": A.Schemes(time=A.Euler)}
    if keq:
        schemes["k"] = A.Schemes(time=A.Euler, divergence=A.Linear)
    if U0 is None:
        U0 = fourier_field(mesh, seed=0)
    if dt is None:
        # dt from CFL = 0.5 with the Courant definition of max_courant_number!
        umag = np.sqrt(np.sum(U0 * U0, axis=0))
        dx = np.power(mesh.cell_volume, 1.0 / 3.0)
        dt = 0.5 * float(np.min(dx / np.maximum(umag, 1e-30)))
    solvers = _solvers(relax_U=1.0, relax_p=1.0, rtol_U=0.1, rtol_p=0.01)
    if keq:
        solvers["k"] = A.SolverSetup(solver=A.Bicgstab(), preconditioner=A.Jacobi(), convergence=1e-7, relax=1.0,
                                     rtol=1e-3)
    config = A.Configuration(solvers=solvers, schemes=schemes,
                             runtime=A.Runtime(iterations=steps, write_interval=-1, time_step=dt),
                             hardware=A.Hardware(backend=A.B200Backend(device=device, precision=precision)),
                             boundaries=BCs)
    model.momentum.U[:] = U0
    A.initialise_(model.momentum.p, 0.0)
    if keq:
        A.initialise_(model.turbulence.k, k0)
    return model, config
