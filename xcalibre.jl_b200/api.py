"""Host-side mirror of XCALibre.jl's user API for the SIMPLE/PISO hot path.

The names, keyword arguments and semantics follow the reference:

  Physics / Fluid{Incompressible} / RANS{Laminar} / LES{Smagorinsky}
      src/ModelPhysics/0_type_definition.jl:196-229, 2_fluid_models.jl:49-71
  Dirichlet, DirichletFunction, Wall, Zerogradient, Extrapolated, Empty,
  Symmetry, Neumann, construct_periodic, assign
      src/Discretise/boundary_conditions/*.jl, Discretise_4_assign_boundaries.jl:5
  Schemes, SolverSetup, Runtime        src/Solve/Solve_1_api.jl:8-211
  Hardware, Configuration              src/Simulate/Simulate_0_types.jl:32-74
  run! -> run_(model, config; pref, ncorrectors, inner_loops)
      src/Solvers/Solvers_3_solver_dispatch.jl:120,225

Everything below the API goes through libxcal_b200.so (``Engine`` classes);
Python only marshals arrays.  ``B200Backend`` is the backend type that
selects this implementation (the reference's ``CUDABackend()`` slot).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Callable

import numpy as np

from . import _abi
from ._lib import check, lib
from .foam import Mesh3

EPS64 = float(np.finfo(np.float64).eps)

# ---------------------------------------------------------------------------
# schemes, solvers, preconditioners (marker types)
# ---------------------------------------------------------------------------


class SteadyState: ...


class Euler: ...


class Linear: ...


class Upwind: ...


class LUST: ...


class Gauss: ...


class Midpoint: ...


@dataclass
class CellBased:
    """Cell-based gradient limiter (Calculate_0_gradient_cell_limiter.jl):
    level 1 = full limiting, 0 = none."""
    level: float = 1.0

    def __post_init__(self):
        if not 0.0 <= float(self.level) <= 1.0:
            raise ValueError(f"CellBased limiter: `level` must be between 0 and 1, got {self.level}")


class FaceBased:
    """Face-based gradient limiter (Calculate_0_gradient_face_limiter.jl):
    per cell the smallest ratio over its internal faces, bounds widened by
    the two cells' difference; FaceBased(mesh) as in the reference (the mesh
    argument is not needed)."""

    def __init__(self, *a, **k):
        pass


class MFaceBased:
    """The modified face-based limiter (Calculate_0_gradient_mface_limiter.jl):
    each internal face corrects both cells' gradients toward the face's value
    bounds in turn.  Applied per cell in ascending face order, which is the
    reference's kernel run on one thread (its parallel runs race on cells
    that share faces); MFaceBased(mesh) as in the reference."""

    def __init__(self, *a, **k):
        pass


class Cg: ...


class Bicgstab: ...


class Jacobi: ...


class DILU: ...


class Steady: ...


class Transient: ...


class Laminar: ...


class Smagorinsky: ...


class KEquation:
    """LES{KEquation} (LES_KEquation.jl): a subgrid kinetic energy
    equation; nut = ck Delta sqrt(k)."""


class KOmega:
    """RANS{KOmega} (RANS_kOmega.jl): k and omega transport equations,
    nut = k / omega."""


class KOmegaSST:
    """RANS{KOmegaSST} (RANS_kOmegaSST.jl): k-omega with F1/F2 blending from
    the wall distance, cross-diffusion and a limited nut."""


class KOmegaLKE:
    """RANS{KOmegaLKE} (RANS_kOmegaLKE.jl): k-omega with a laminar kinetic
    energy kl and an intermittency trigger for transition; needs Tu (the
    freestream turbulence intensity) and the wall patches."""


class Incompressible: ...


class Isothermal: ...


def _inst(x):
    return x() if isinstance(x, type) else x


@dataclass
class Schemes:
    time: type = SteadyState
    divergence: type = Linear
    laplacian: type = Linear
    gradient: type = Gauss
    limiter: object = None


class JacobiSmoother:
    """JacobiSmoother (Smoothers_jacobi.jl:26-51): ``loops`` weighted Jacobi
    sweeps, weight ``omega``, applied to the field before each Krylov solve
    (solve_system!, Solve_1_api.jl:284).  Constructors as the reference's:
    ``JacobiSmoother(mesh)`` (5 loops, omega 1),
    ``JacobiSmoother(domain=mesh, loops=n, omega=2/3)`` and
    ``JacobiSmoother(loops, omega, x_temp)``."""

    def __init__(self, *args, domain=None, loops=None, omega=None):
        if len(args) == 1:
            domain, loops, omega = args[0], 5, 1.0
        elif len(args) >= 2:
            loops, omega = args[0], args[1]
        elif domain is None or loops is None:
            raise TypeError("JacobiSmoother(mesh), JacobiSmoother(domain=, loops=[, omega=]) or "
                            "JacobiSmoother(loops, omega, x_temp)")
        elif omega is None:
            omega = 2.0 / 3.0
        self.loops = int(loops)
        self.omega = float(omega)
        if self.loops < 0:
            raise ValueError("JacobiSmoother: loops must be >= 0")


@dataclass
class SolverSetup:
    solver: object
    preconditioner: object
    convergence: float
    relax: float
    float_type: str = "Float64"
    smoother: object = None
    limit: object = None
    itmax: int = 1000
    atol: float | None = None
    rtol: float = 0.1

    def __post_init__(self):
        if self.atol is None:
            self.atol = EPS64 ** 0.9  # (eps(float_type))^0.9 (Solve_1_api.jl:70)
        if self.smoother is not None and not isinstance(self.smoother, JacobiSmoother):
            raise NotImplementedError("JacobiSmoother is the only smoother")


@dataclass
class Runtime:
    iterations: int
    write_interval: int
    time_step: float
    adaptive: object = None


@dataclass
class B200Backend:
    """Backend selecting libxcal_b200 (one GPU).  ``precision`` is "fp64"
    (plain path) or "mixed" (FP32 Krylov inner solves inside an FP64 defect
    correction; each inner solve reduces its residual by ``inner_rtol`` at
    most, never past the FP64 path's own stopping target)."""
    device: int = 0
    precision: str = "fp64"
    inner_rtol: float = 1e-3


@dataclass
class Hardware:
    backend: object
    workgroup: int = 32


@dataclass
class Configuration:
    solvers: dict
    schemes: dict
    runtime: Runtime
    hardware: Hardware
    boundaries: dict
    postprocess: object = None


# ---------------------------------------------------------------------------
# physics
# ---------------------------------------------------------------------------


@dataclass
class Fluid:
    kind: type
    nu: float
    rho: float = 1.0


@dataclass
class RANS:
    """RANS{Laminar}, RANS{KOmega}(; beta+, alpha1, beta1, sigma_k,
    sigma_omega) (RANS_kOmega.jl:29-33) or RANS{KOmegaSST}(; beta+, alpha1,
    sigma_k1, sigma_k2, sigma_omega1, sigma_omega2, beta1, beta2, kappa,
    walls) (RANS_kOmegaSST.jl:57-61) or RANS{KOmegaLKE}(; Tu, walls)
    (RANS_kOmegaLKE.jl:60-64, its other coefficients fixed); unset
    coefficients take the model's defaults."""
    model: type = Laminar
    beta_star: float | None = None
    alpha1: float | None = None
    beta1: float | None = None
    sigma_k: float | None = None
    sigma_omega: float | None = None
    beta2: float | None = None
    sigma_k1: float | None = None
    sigma_k2: float | None = None
    sigma_omega1: float | None = None
    sigma_omega2: float | None = None
    kappa: float | None = None
    walls: list | None = None
    Tu: float | None = None

    def coeffs(self) -> dict:
        if self.model is KOmegaSST:
            d = dict(beta_star=0.09, alpha1=0.31, sigma_k1=0.85, sigma_k2=1.0, sigma_omega1=0.5, sigma_omega2=0.856,
                     beta1=0.075, beta2=0.0828, kappa=0.41)
        else:
            d = dict(beta_star=0.09, alpha1=0.52, beta1=0.072, sigma_k=0.5, sigma_omega=0.5)
        for k in list(d):
            v = getattr(self, k, None)
            if v is not None:
                d[k] = float(v)
        return d


@dataclass
class LES:
    """LES{Smagorinsky}(; C) (LES_Smagorinsky.jl) or LES{KEquation}(; ck,
    ce) (LES_KEquation.jl:35-39)."""
    model: type = Smagorinsky
    C: float = 0.15
    ck: float = 0.094
    ce: float = 1.048


@dataclass
class Energy:
    kind: type = Isothermal


@dataclass
class Momentum:
    U: np.ndarray
    p: np.ndarray


class Physics:
    def __init__(self, time, fluid: Fluid, turbulence, energy, domain: Mesh3):
        self.time = _inst(time)
        self.fluid = fluid
        self.turbulence = turbulence
        self.energy = energy
        self.domain = domain
        n = domain.n_cells
        self.momentum = Momentum(U=np.zeros((3, n)), p=np.zeros(n))
        self.nut = np.zeros(n)
        # model.turbulence.k / .omega / .nut, as the reference's fields
        if isinstance(turbulence, (RANS, LES)):
            turbulence.nut = self.nut
            if isinstance(turbulence, RANS) and turbulence.model in (KOmega, KOmegaSST, KOmegaLKE):
                turbulence.k = np.zeros(n)
                turbulence.omega = np.zeros(n)
            if isinstance(turbulence, LES) and turbulence.model is KEquation:
                turbulence.k = np.zeros(n)
            if isinstance(turbulence, RANS) and turbulence.model is KOmegaLKE:
                turbulence.kl = np.zeros(n)
            if isinstance(turbulence, RANS) and turbulence.model in (KOmegaSST, KOmegaLKE):
                turbulence.y = np.zeros(n)


def initialise_(field: np.ndarray, value) -> None:
    """initialise! (src/Fields/Fields_0_types.jl:381-401)."""
    if field.ndim == 2:
        v = np.asarray(value, dtype=np.float64)
        if v.shape != (3,):
            raise ValueError("Vectors should have 3 components")
        field[:] = v[:, None]
    else:
        field[:] = float(value)


# ---------------------------------------------------------------------------
# boundary conditions
# ---------------------------------------------------------------------------


@dataclass
class BC:
    kind: int
    name: str
    value: object = 0.0
    func: Callable | None = None
    face_map: np.ndarray | None = None
    distance: np.ndarray | None = None
    partner: str | None = None
    wall: tuple | None = None  # wall functions: (kappa, beta1, cmu^0.25, yPlusLam, E)


def Dirichlet(name, value):
    return BC(_abi.BC_DIRICHLET, name, value)


def DirichletFunction(name, f):
    """``f(coords, time, index)`` returns a 3-vector (vector fields) or a
    number (scalar fields); it is evaluated on the host for every face."""
    return BC(_abi.BC_DIRICHLET_FUNCTION, name, 0.0, func=f)


def Wall(name, value=0.0):
    return BC(_abi.BC_WALL, name, value)


def Zerogradient(name):
    return BC(_abi.BC_ZEROGRADIENT, name)


def Extrapolated(name, value=0.0):
    """Extrapolated(name[, value]) (extrapolated.jl:12-20): zero gradient,
    semi-implicitly; the value is stored but not used, as in the reference."""
    return BC(_abi.BC_EXTRAPOLATED, name, value)


def y_plus_laminar(E: float, kappa: float) -> float:
    """y_plus_laminar (RANS_functions.jl:42-45)."""
    yL = 11.0
    for _ in range(10):
        yL = math.log(max(yL * E, 1.0)) / kappa
    return yL


def _wall_consts(kappa, beta1, cmu, E):
    return (float(kappa), float(beta1), float(cmu) ** 0.25, y_plus_laminar(float(E), float(kappa)), float(E))


def OmegaWallFunction(name, kappa=0.41, beta1=0.075, cmu=0.09, B=5.2, E=9.8):
    """OmegaWallFunction (Discretise_0_types.jl:83-113): the wall cell's
    omega fixed to omega_log or omega_vis by y+ (constrain!)."""
    return BC(_abi.BC_OMEGA_WALL, name, 0.0, wall=_wall_consts(kappa, beta1, cmu, E))


def KWallFunction(name, kappa=0.41, beta1=0.075, cmu=0.09, B=5.2, E=9.8):
    """KWallFunction (Discretise_0_types.jl:39-66): zero gradient for k, and
    the wall cell's production from the log law (set_production!,
    RANS_functions.jl:66-117)."""
    return BC(_abi.BC_K_WALL, name, 0.0, wall=_wall_consts(kappa, beta1, cmu, E))


def NutWallFunction(name, kappa=0.41, beta1=0.075, cmu=0.09, B=5.2, E=9.8):
    """NutWallFunction: zero gradient for nut, and the wall face's nutf from
    the log law (correct_nut_wall!, RANS_functions.jl:119-172)."""
    return BC(_abi.BC_NUT_WALL, name, 0.0, wall=_wall_consts(kappa, beta1, cmu, E))


def Empty(name):
    return BC(_abi.BC_EMPTY, name)


def Symmetry(name):
    return BC(_abi.BC_SYMMETRY, name)


def Neumann(name, value):
    return BC(_abi.BC_NEUMANN, name, value)


def _pairwise_sum(a: np.ndarray) -> np.ndarray:
    """Julia's `sum` over a vector (pairwise blocks of 1024, sequential leaves)."""
    def rec(lo, hi):
        if lo == hi:
            return a[lo].copy()
        if hi - lo < 1024:
            v = a[lo] + a[lo + 1]
            for i in range(lo + 2, hi + 1):
                v = v + a[i]
            return v
        mid = lo + ((hi - lo) >> 1)
        return rec(lo, mid) + rec(mid + 1, hi)
    return rec(0, a.shape[0] - 1)


def construct_periodic(mesh: Mesh3, backend, patch1: str, patch2: str, tol: float = 1e-7):
    """construct_periodic (src/Discretise/boundary_conditions/periodic.jl:95-217):
    match the faces of two conformal patches by translated centroids."""
    r1, r2 = mesh.patch_range(patch1), mesh.patch_range(patch2)
    if len(r1) != len(r2):
        raise ValueError(f"Periodic mismatch: Patch {patch1} has {len(r1)} faces, but {patch2} has {len(r2)}")
    c1 = mesh.face_centre[r1.start:r1.stop]
    c2 = mesh.face_centre[r2.start:r2.stop]
    nf = len(r1)
    tr = _pairwise_sum(c2) / float(nf) - _pairwise_sum(c1) / float(nf)
    targets = c1 + tr
    # lexicographic extremes (minimum/maximum over SVectors)
    order = np.lexsort((targets[:, 2], targets[:, 1], targets[:, 0]))
    ext = targets[order[-1]] - targets[order[0]]
    axis = int(np.argmax(ext))
    p1 = np.argsort(targets[:, axis], kind="stable")
    p2 = np.argsort(c2[:, axis], kind="stable")
    ts, ss = targets[p1], c2[p2]
    map1 = np.zeros(nf, dtype=np.int32)
    map2 = np.zeros(nf, dtype=np.int32)
    start = 0
    sv = ss[:, axis]
    for i in range(nf):
        t = ts[i]
        tv = t[axis]
        while start < nf and sv[start] < tv - tol:
            start += 1
        stop = start
        while stop < nf and sv[stop] - tv <= tol:
            stop += 1
        if stop == start:
            raise ValueError(f"Periodic mismatch at Face {i}: no match found closer than tolerance {tol}")
        d = ss[start:stop] - t
        dist = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
        j = int(np.argmin(dist))
        if not dist[j] < tol:
            raise ValueError(f"Periodic mismatch at Face {i}: no match found closer than tolerance {tol}")
        l1, l2 = p1[i], p2[start + j]
        map1[l1] = r2.start + l2
        map2[l2] = r1.start + l1
    parent = BC(_abi.BC_PERIODIC_PARENT, patch1, 0.0, face_map=map1, distance=tr, partner=patch2)
    shadow = BC(_abi.BC_PERIODIC, patch2, 0.0, face_map=map2, distance=tr, partner=patch1)
    return parent, shadow


def assign(region: Mesh3, **fields) -> dict:
    """assign (src/Discretise/Discretise_4_assign_boundaries.jl:5-18)."""
    out = {}
    nb = len(region.patch_names)
    for name, bcs in fields.items():
        bcs = list(bcs)
        for bc in bcs:
            region.patch_index(bc.name)  # raises for unknown names
        if len(bcs) != nb:
            raise ValueError(f"Inconsistent number of boundaries assigned to field {name}")
        out[name] = bcs
    return out


# ---------------------------------------------------------------------------
# engine: handles of the C ABI
# ---------------------------------------------------------------------------


class Context:
    def __init__(self, device: int = 0):
        h = C.c_void_p()
        code = lib().xcal_ctx_create(device, C.byref(h))
        if code != 0:
            raise RuntimeError(f"xcal_ctx_create failed ({code}); is a CUDA device visible?")
        self.h = h

    def close(self):
        if self.h:
            lib().xcal_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceMesh:
    def __init__(self, ctx: Context, mesh: Mesh3):
        self.ctx, self.mesh = ctx, mesh
        desc, keep = _abi.mesh_desc(mesh)
        h = C.c_void_p()
        check(lib().xcal_mesh_upload(ctx.h, C.byref(desc), C.byref(h)), ctx.h)
        self.h = h

    def close(self):
        if self.h:
            lib().xcal_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _bc_array(mesh: Mesh3, bcs, ncomp: int, keep: list):
    arr = (_abi.BCDesc * max(1, len(bcs)))()
    for k, bc in enumerate(bcs):
        d = arr[k]
        d.type = bc.kind
        d.patch = mesh.patch_index(bc.name)
        v = np.zeros(3)
        if bc.kind not in (_abi.BC_DIRICHLET_FUNCTION, _abi.BC_PERIODIC, _abi.BC_PERIODIC_PARENT):
            val = np.asarray(bc.value, dtype=np.float64).ravel()
            v[: val.size] = val[:3]
        for c in range(3):
            d.value[c] = v[c]
        if bc.kind == _abi.BC_DIRICHLET_FUNCTION:
            vals = dirichlet_function_values(mesh, bc, ncomp, 0.0)
            keep.append(vals)
            d.face_values = _abi.ptr(vals, C.c_double)
        if bc.face_map is not None:
            fm = np.ascontiguousarray(bc.face_map, dtype=np.int32)
            keep.append(fm)
            d.face_map = _abi.ptr(fm, C.c_int32)
            for c in range(3):
                d.distance[c] = float(bc.distance[c])
            d.partner_patch = mesh.patch_index(bc.partner)
        if bc.wall is not None:
            for c in range(5):
                d.wall[c] = float(bc.wall[c])
    return arr


def dirichlet_function_values(mesh: Mesh3, bc: BC, ncomp: int, time) -> np.ndarray:
    """Evaluate f(face.centre, time, i) for every face of the patch (i is the
    1-based local face index, as in dirichletFunction.jl)."""
    r = mesh.patch_range(bc.name)
    vals = np.zeros((len(r), ncomp))
    for i, f in enumerate(r):
        v = bc.func(mesh.face_centre[f], time, i + 1)
        vals[i] = np.asarray(v, dtype=np.float64).ravel()[:ncomp]
    return np.ascontiguousarray(vals.ravel())


_SCHEME_TIME = {SteadyState: _abi.TIME_STEADY, Euler: _abi.TIME_EULER}
_SCHEME_DIV = {Linear: _abi.DIV_LINEAR, Upwind: _abi.DIV_UPWIND, LUST: _abi.DIV_LUST}
_SCHEME_GRAD = {Gauss: _abi.GRAD_GAUSS, Midpoint: _abi.GRAD_MIDPOINT}


def _kind(x):
    return x if isinstance(x, type) else type(x)


def _limiter(lim):
    if lim is None:
        return _abi.LIMITER_NONE, 0.0
    if isinstance(lim, CellBased):
        return _abi.LIMITER_CELL, float(lim.level)
    if _kind(lim) is FaceBased:
        return _abi.LIMITER_FACE, 0.0
    if _kind(lim) is MFaceBased:
        return _abi.LIMITER_MFACE, 0.0
    raise NotImplementedError(f"unknown gradient limiter {lim!r} (CellBased, FaceBased, MFaceBased)")


def _solver_desc(s: SolverSetup) -> _abi.SolverSetupDesc:
    solver = {Cg: _abi.SOLVER_CG, Bicgstab: _abi.SOLVER_BICGSTAB}[_kind(s.solver)]
    pre = {Jacobi: _abi.PRECOND_JACOBI, DILU: _abi.PRECOND_DILU, type(None): _abi.PRECOND_NONE}[_kind(s.preconditioner)]
    sm = s.smoother
    return _abi.SolverSetupDesc(solver=solver, precond=pre, convergence=float(s.convergence),
                                relax=float(s.relax), atol=float(s.atol), rtol=float(s.rtol), itmax=int(s.itmax),
                                smoother_loops=sm.loops if sm is not None else 0,
                                smoother_omega=sm.omega if sm is not None else 0.0)


def delta_scaling(mesh: Mesh3, bcs) -> tuple[float, float]:
    """delta_scaling(mesh::Mesh3, BCs) (LES_functions.jl:33-56): for the first
    Empty BC, (|pmin.n| + |pmax.n|, 0.5), n the normal of the patch's first
    face and pmin/pmax the bounding box (started at the origin) of the
    boundary faces' nodes (bounding_box, Mesh_1_functions.jl:70-100); with no
    Empty BC (1, 1/3).  A 2D mesh (Mesh2): (1, 0.5) (:28-31)."""
    if getattr(mesh, "dim", 3) == 2:
        return 1.0, 0.5
    for bc in bcs:
        if bc.kind != _abi.BC_EMPTY:
            continue
        pm = mesh.polymesh
        if pm is not None:
            off = np.asarray(pm.face_offsets)
            nI = int(np.asarray(pm.neighbour).size)
            nodes = np.asarray(pm.face_nodes)[off[nI]:off[-1]]
            pts = np.asarray(pm.points, dtype=np.float64)[nodes]
        else:  # no node data: the boundary-face centres
            pts = np.asarray(mesh.face_centre, dtype=np.float64)[:mesh.n_bfaces]
        pmin = np.minimum(pts.min(axis=0), 0.0)
        pmax = np.maximum(pts.max(axis=0), 0.0)
        n = np.asarray(mesh.face_normal, dtype=np.float64)[mesh.patch_range(bc.name).start]
        d1 = abs(pmin[0] * n[0] + pmin[1] * n[1] + pmin[2] * n[2])
        d2 = abs(pmax[0] * n[0] + pmax[1] * n[1] + pmax[2] * n[2])
        return float(d1 + d2), 0.5
    return 1.0, 1.0 / 3.0


def build_config(model: Physics, config: Configuration, pref=None, inner_loops=None, ncorrectors: int = 0):
    """Translate the Python API objects into an xcal_config (keep the second
    return value alive while the config is in use).  ncorrectors: SIMPLE
    non-orthogonal correctors (run!(...; ncorrectors))."""
    mesh = model.domain
    keep: list = []
    transient = isinstance(model.time, Transient)
    turb = model.turbulence
    les = isinstance(turb, LES)
    keq = les and turb.model is KEquation
    sst = isinstance(turb, RANS) and turb.model is KOmegaSST
    lke = isinstance(turb, RANS) and turb.model is KOmegaLKE
    kw = isinstance(turb, RANS) and turb.model in (KOmega, KOmegaSST, KOmegaLKE)
    if lke and turb.Tu is None:
        raise ValueError("RANS{KOmegaLKE} needs Tu (RANS_kOmegaLKE.jl:60)")
    bnd = config.boundaries
    bU = _bc_array(mesh, bnd["U"], 3, keep)
    bP = _bc_array(mesh, bnd["p"], 1, keep)
    nut_bcs = bnd.get("nut", []) if (les or kw) else []
    bN = _bc_array(mesh, nut_bcs, 1, keep)
    k_bcs = bnd.get("k", []) if (kw or keq) else []
    w_bcs = bnd.get("omega", []) if kw else []
    kl_bcs = bnd.get("kl", []) if lke else []
    bK = _bc_array(mesh, k_bcs, 1, keep)
    bW = _bc_array(mesh, w_bcs, 1, keep)
    bKl = _bc_array(mesh, kl_bcs, 1, keep)
    # wall_distance! (Calculate_4_wall_distance.jl:12-27): per BC of the
    # first field, Dirichlet 0 on the walls, Empty, else Extrapolated
    y_bcs = []
    if sst or lke:
        walls = list(turb.walls or [])
        for bc in next(iter(bnd.values())):
            if bc.name in walls:
                y_bcs.append(Dirichlet(bc.name, 0.0))
            elif bc.kind == _abi.BC_EMPTY:
                y_bcs.append(Empty(bc.name))
            else:
                y_bcs.append(Extrapolated(bc.name))
    bY = _bc_array(mesh, y_bcs, 1, keep)
    keep += [bU, bP, bN, bK, bW, bY, bKl]
    sY = config.schemes.get("y", Schemes()) if (sst or lke) else Schemes()
    slv_y = _solver_desc(config.solvers["y"]) if (sst or lke) else _abi.SolverSetupDesc()
    sKl = config.schemes.get("kl", Schemes()) if lke else Schemes()
    slv_kl = _solver_desc(config.solvers["kl"]) if lke else _abi.SolverSetupDesc()
    co = turb.coeffs() if (kw and not lke) else {}
    sK = config.schemes.get("k", Schemes()) if (kw or keq) else Schemes()
    sW = config.schemes.get("omega", Schemes()) if kw else Schemes()
    slv_k = _solver_desc(config.solvers["k"]) if (kw or keq) else _abi.SolverSetupDesc()
    slv_w = _solver_desc(config.solvers["omega"]) if kw else _abi.SolverSetupDesc()
    sU, sP = config.schemes["U"], config.schemes["p"]
    backend = config.hardware.backend
    prec = _abi.PREC_MIXED if getattr(backend, "precision", "fp64") == "mixed" else _abi.PREC_FP64
    if inner_loops is None:
        inner_loops = 2 if transient else 0
    # delta! reads config.boundaries[1] (LES_functions.jl:7): the first field's BCs
    dist, power = delta_scaling(mesh, next(iter(bnd.values()))) if les else (1.0, 1.0 / 3.0)
    cfg = _abi.ConfigDesc(
        algorithm=_abi.ALGO_PISO if transient else _abi.ALGO_SIMPLE,
        turbulence=(_abi.TURB_KEQUATION if keq else _abi.TURB_SMAGORINSKY if les else _abi.TURB_KOMEGA_SST if sst
                    else _abi.TURB_KOMEGA_LKE if lke else _abi.TURB_KOMEGA if kw else _abi.TURB_LAMINAR),
        nu=float(model.fluid.nu), smagorinsky_C=float(turb.C) if (les and not keq) else 0.0,
        les_delta_distance=dist, les_delta_power=power,
        U_schemes=_abi.SchemesDesc(time=_SCHEME_TIME[_kind(sU.time)], divergence=_SCHEME_DIV[_kind(sU.divergence)],
                                   gradient=_SCHEME_GRAD[_kind(sU.gradient)], limiter=_limiter(sU.limiter)[0],
                                   limiter_level=_limiter(sU.limiter)[1]),
        p_schemes=_abi.SchemesDesc(time=_SCHEME_TIME[_kind(sP.time)], divergence=_SCHEME_DIV[_kind(sP.divergence)],
                                   gradient=_SCHEME_GRAD[_kind(sP.gradient)], limiter=_limiter(sP.limiter)[0],
                                   limiter_level=_limiter(sP.limiter)[1]),
        U_solver=_solver_desc(config.solvers["U"]), p_solver=_solver_desc(config.solvers["p"]),
        iterations=int(config.runtime.iterations), dt=float(config.runtime.time_step),
        has_pref=0 if pref is None else 1, pref=0.0 if pref is None else float(pref),
        inner_loops=int(inner_loops), ncorrectors=int(ncorrectors), precision=prec,
        inner_rtol=float(getattr(backend, "inner_rtol", 1e-3)),
        n_bc_U=len(bnd["U"]), n_bc_p=len(bnd["p"]), n_bc_nut=len(nut_bcs),
        bc_U=C.cast(bU, C.POINTER(_abi.BCDesc)), bc_p=C.cast(bP, C.POINTER(_abi.BCDesc)),
        bc_nut=C.cast(bN, C.POINTER(_abi.BCDesc)),
        kw_beta_star=co.get("beta_star", 0.0), kw_alpha1=co.get("alpha1", 0.0), kw_beta1=co.get("beta1", 0.0),
        kw_sigma_k=co.get("sigma_k1" if sst else "sigma_k", 0.0),
        kw_sigma_omega=co.get("sigma_omega1" if sst else "sigma_omega", 0.0),
        sst_beta2=co.get("beta2", 0.0), sst_sigma_k2=co.get("sigma_k2", 0.0),
        sst_sigma_omega2=co.get("sigma_omega2", 0.0),
        y_schemes=_abi.SchemesDesc(gradient=_SCHEME_GRAD[_kind(sY.gradient)]), y_solver=slv_y, n_bc_y=len(y_bcs),
        bc_y=C.cast(bY, C.POINTER(_abi.BCDesc)),
        k_schemes=_abi.SchemesDesc(time=_SCHEME_TIME[_kind(sK.time)], divergence=_SCHEME_DIV[_kind(sK.divergence)],
                                   gradient=_SCHEME_GRAD[_kind(sK.gradient)]),
        omega_schemes=_abi.SchemesDesc(time=_SCHEME_TIME[_kind(sW.time)],
                                       divergence=_SCHEME_DIV[_kind(sW.divergence)]),
        k_solver=slv_k, omega_solver=slv_w, n_bc_k=len(k_bcs), n_bc_omega=len(w_bcs),
        bc_k=C.cast(bK, C.POINTER(_abi.BCDesc)), bc_omega=C.cast(bW, C.POINTER(_abi.BCDesc)),
        keq_ck=float(turb.ck) if keq else 0.0, keq_ce=float(turb.ce) if keq else 0.0,
        lke_Tu=float(turb.Tu) if lke else 0.0,
        kl_schemes=_abi.SchemesDesc(time=_SCHEME_TIME[_kind(sKl.time)], divergence=_SCHEME_DIV[_kind(sKl.divergence)],
                                    gradient=_SCHEME_GRAD[_kind(sKl.gradient)]),
        kl_solver=slv_kl, n_bc_kl=len(kl_bcs), bc_kl=C.cast(bKl, C.POINTER(_abi.BCDesc)))
    return cfg, keep


class Case:
    """A solver case on the GPU (xcal_case)."""

    def __init__(self, dmesh: DeviceMesh, cfg: _abi.ConfigDesc):
        self.dmesh, self.ctx = dmesh, dmesh.ctx
        self.mesh = dmesh.mesh
        self.komega = cfg.turbulence in (_abi.TURB_KOMEGA, _abi.TURB_KOMEGA_SST, _abi.TURB_KOMEGA_LKE)
        self.lke = cfg.turbulence == _abi.TURB_KOMEGA_LKE
        self.kequation = cfg.turbulence == _abi.TURB_KEQUATION
        h = C.c_void_p()
        check(lib().xcal_case_create(self.ctx.h, dmesh.h, C.byref(cfg), C.byref(h)), self.ctx.h)
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().xcal_case_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, code):
        check(code, self.ctx.h)

    def _size(self, field):
        nc, kind = _abi.FIELD_SHAPE[field]
        per = self.mesh.n_cells if kind == "cell" else self.mesh.n_faces
        return nc, per

    def set_field(self, field: int, values) -> None:
        nc, per = self._size(field)
        a = np.ascontiguousarray(np.asarray(values, dtype=np.float64).reshape(nc * per))
        self._chk(lib().xcal_case_set_field(self.h, field, _abi.ptr(a, C.c_double), a.size))

    def get_field(self, field: int, out: np.ndarray | None = None) -> np.ndarray:
        """The field in original cell/face order ([components, n] for vectors).
        out: a C-contiguous float64 array of that size to write into (e.g. a
        pinned host buffer, which the device copies into directly)."""
        nc, per = self._size(field)
        if out is not None:
            if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != nc * per:
                raise ValueError("get_field: out must be C-contiguous float64 with %d values" % (nc * per))
            a = out.reshape(nc * per)
        else:
            a = np.empty(nc * per)
        self._chk(lib().xcal_case_get_field(self.h, field, _abi.ptr(a, C.c_double), a.size))
        if out is not None:
            return out
        return a.reshape(nc, per) if nc > 1 else a

    def nnz(self, eqn: int) -> int:
        n = C.c_int64()
        self._chk(lib().xcal_case_nnz(self.h, eqn, C.byref(n)))
        return n.value

    def pattern(self, eqn: int):
        nnz = self.nnz(eqn)
        rp = np.empty(self.mesh.n_cells + 1, dtype=np.int32)
        cv = np.empty(nnz, dtype=np.int32)
        self._chk(lib().xcal_case_csr_pattern(self.h, eqn, _abi.ptr(rp, C.c_int32), _abi.ptr(cv, C.c_int32)))
        return rp, cv

    def system(self, eqn: int, component: int = 0):
        nz = np.empty(self.nnz(eqn))
        b = np.empty(self.mesh.n_cells)
        self._chk(lib().xcal_case_get_system(self.h, eqn, component, _abi.ptr(nz, C.c_double),
                                             _abi.ptr(b, C.c_double)))
        return nz, b

    def simple_iterate(self, n: int):
        res = np.zeros((max(n, 1), 4))
        done, conv = C.c_int32(), C.c_int32()
        self._chk(lib().xcal_simple_iterate(self.h, n, _abi.ptr(res, C.c_double), C.byref(done), C.byref(conv)))
        return res[: done.value], bool(conv.value)

    def piso_step(self, n: int):
        res = np.zeros((max(n, 1), 4))
        co = np.zeros(max(n, 1))
        done = C.c_int32()
        self._chk(lib().xcal_piso_step(self.h, n, _abi.ptr(res, C.c_double), _abi.ptr(co, C.c_double),
                                       C.byref(done)))
        return res[: done.value], co[: done.value]

    # fine-grained hooks
    def initial_calculations(self):
        self._chk(lib().xcal_initial_calculations(self.h))

    def discretise(self, eqn):
        self._chk(lib().xcal_discretise(self.h, eqn))

    def apply_boundary_conditions(self, eqn, comp=0):
        self._chk(lib().xcal_apply_boundary_conditions(self.h, eqn, comp))

    def implicit_relaxation_diagdom(self, comp):
        self._chk(lib().xcal_implicit_relaxation_diagdom(self.h, comp))

    def set_reference(self):
        self._chk(lib().xcal_set_reference(self.h))

    def update_preconditioner(self, eqn):
        self._chk(lib().xcal_update_preconditioner(self.h, eqn))

    def solve_system(self, eqn, comp=0):
        r, it = C.c_double(), C.c_int32()
        self._chk(lib().xcal_solve_system(self.h, eqn, comp, C.byref(r), C.byref(it)))
        return r.value, it.value

    def solve_equation(self, eqn):
        res = np.zeros(3)
        self._chk(lib().xcal_solve_equation(self.h, eqn, _abi.ptr(res, C.c_double)))
        return res if eqn == _abi.EQN_U else res[0]

    def pressure_predictor(self):
        self._chk(lib().xcal_pressure_predictor(self.h))

    def flux_divergence(self):
        self._chk(lib().xcal_flux_divergence(self.h))

    def explicit_relaxation_p(self, alpha):
        self._chk(lib().xcal_explicit_relaxation_p(self.h, float(alpha)))

    def grad_p(self):
        self._chk(lib().xcal_grad_p(self.h))

    def correct(self):
        self._chk(lib().xcal_correct(self.h))

    def turbulence(self):
        self._chk(lib().xcal_turbulence(self.h))

    def max_courant(self):
        c = C.c_double()
        self._chk(lib().xcal_max_courant(self.h, C.byref(c)))
        return c.value

    def timings(self):
        ms = np.zeros(6)
        lib().xcal_get_timings(self.h, _abi.ptr(ms, C.c_double), 6)
        return ms

    def stream(self) -> int:
        s = C.c_void_p()
        self._chk(lib().xcal_case_stream(self.h, C.byref(s)))
        return s.value or 0

    def set_profiling(self, on: bool = True):
        self._chk(lib().xcal_case_set_profiling(self.h, 1 if on else 0))

    def tuning(self) -> dict:
        """Launch shapes chosen by the autotuner (tuning runs now if it has
        not yet): per equation the BiCGSTAB SpMV rows per thread (0 = tile
        kernel) and block size, and the DILU form (one-block sweeps, or one
        cooperative launch over every level)."""
        a = np.zeros(6, dtype=np.int32)
        self._chk(lib().xcal_case_tuning(self.h, _abi.ptr(a, C.c_int32)))
        return {eq: {"spmv_rows_per_thread": int(a[3 * k]), "spmv_block": int(a[3 * k + 1]),
                     "dilu_one_block": bool(a[3 * k + 2] == 1), "dilu_grid": bool(a[3 * k + 2] == 2)}
                for k, eq in enumerate(("U", "p"))}

    def set_dilu_mode(self, mode: int):
        """0 = autotuned, 1 = one-block sweeps, 2 = per-level kernels,
        3 = every level in one cooperative launch (same results)."""
        self._chk(lib().xcal_case_set_dilu_mode(self.h, int(mode)))

    def solve_report(self) -> dict:
        """Last Krylov solve of each system (Ux, Uy, Uz, p, k, omega, wall
        distance): iterations and status (0 running, 1 solved, 2 stopped at
        itmax, 3 zero curvature, 4 breakdown, 5 zero right-hand side), and
        how many solves since creation stopped at itmax."""
        it = np.zeros(7, dtype=np.int32)
        st = np.zeros(7, dtype=np.int32)
        hits = C.c_int64()
        self._chk(lib().xcal_case_solve_report(self.h, _abi.ptr(it, C.c_int32), _abi.ptr(st, C.c_int32),
                                               C.byref(hits)))
        return {"iterations": it, "status": st, "itmax_hits": int(hits.value)}

    def set_inner_cg(self, mode: int):
        """Mixed precision, CG + Jacobi inner solves: 0 = on the Jacobi-scaled
        system (default), 1 = the FP32 form of the FP64 path's kernels,
        2 + s + 4 g + 8 w = the scaled-system kernel in launch shape s (0..3:
        768/1024 threads, with or without early loads of the next row's
        slots), with x and p in global memory (g = 1) and per-slice slot
        widths (w = 1).  Shapes with the same thread count, g and w give the
        same results bit for bit."""
        self._chk(lib().xcal_case_set_inner_cg(self.h, int(mode)))

    def checkpoint(self) -> dict:
        """The case's state as host arrays (every field the ABI reads: U, p,
        face mass flux, face velocity and pressure, nu_eff, gradients, rD,
        H...): with ``restore`` a new case on the same mesh and configuration
        continues exactly as this one would."""
        return {name: self.get_field(getattr(_abi, name)).copy() for name in self._state_fields()}

    def _state_fields(self) -> tuple:
        extra = KOMEGA_FIELDS if self.komega else ("FIELD_K",) if self.kequation else ()
        return CHECKPOINT_FIELDS + extra + (("FIELD_KL",) if self.lke else ())

    def restore(self, state: dict) -> None:
        """Set the fields of a ``checkpoint`` and mark the state complete, so
        the next iteration does not redo the run's initial calculations."""
        for name in self._state_fields():
            if name in state:
                self.set_field(getattr(_abi, name), state[name])
        self._chk(lib().xcal_case_mark_initialised(self.h))

    def set_persistent(self, on=True):
        """Persistent CG (one launch per solve): False / True, or 2 (the
        cluster form only), 256 / 512 / 1024 (that cooperative block form
        only), 4 / 5 (one block of 1024 / 512 threads per SM owning every
        G-th tile).  Same results in every form."""
        mode = int(on) if isinstance(on, bool) else int(on)
        self._chk(lib().xcal_case_set_persistent(self.h, mode))

    def set_graph_mode(self, on: bool = True):
        """Replay each SIMPLE iteration / PISO step as one captured CUDA graph
        (device-driven Krylov loops; same results as the default mode)."""
        self._chk(lib().xcal_case_set_graph_mode(self.h, 1 if on else 0))

    def profile(self, which: int):
        """(summed device ms, timed launches) of a kernel class:
        0 = CG SpMV, 1 = BiCGSTAB SpMV, 2 = DILU applications, 3 = CG update;
        4 = (0, every CG SpMV launch that did work); 5 = persistent CG
        launches (ms, CG iterations).  Steady-state chunks run as CUDA graphs
        in which only sampled iterations are timed."""
        ms, n = C.c_double(), C.c_int64()
        self._chk(lib().xcal_case_get_profile(self.h, which, C.byref(ms), C.byref(n)))
        return ms.value, n.value


    def footprint(self) -> tuple[int, int]:
        """(device bytes of the case, device bytes of its mesh)."""
        cb, mb = C.c_int64(), C.c_int64()
        self._chk(lib().xcal_case_footprint(self.h, C.byref(cb), C.byref(mb)))
        return cb.value, mb.value


def footprint_estimate(mesh: Mesh3, precision: str = "fp64", dilu_U: bool = True, dilu_p: bool = False) -> int:
    """Device bytes a case on ``mesh`` will hold (mesh + case), before it is
    created: the admission test of the serving loop."""
    b = C.c_int64()
    check(lib().xcal_footprint_estimate(mesh.n_cells, mesh.n_faces, mesh.n_bfaces,
                                        _abi.PREC_MIXED if precision == "mixed" else _abi.PREC_FP64,
                                        1 if dilu_U else 0, 1 if dilu_p else 0, C.byref(b)), None)
    return b.value


class Batch:
    """Resident batch of steady cases advanced together (xcal_batch_*): each
    Krylov solve is one batched launch sequence over all cases, with
    per-case scalars, so results do not depend on the batch composition."""

    def __init__(self, ctx: Context, max_cases: int, budget_bytes: int):
        self.ctx = ctx
        h = C.c_void_p()
        check(lib().xcal_batch_create(ctx.h, int(max_cases), int(budget_bytes), C.byref(h)), ctx.h)
        self.h = h
        self.cases: list[Case] = []
        self.last_diverged: list[Case] = []

    def close(self):
        if getattr(self, "h", None):
            lib().xcal_batch_destroy(self.h)
            self.h = None
            self.cases = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, case: Case, charge_bytes: int = 0) -> bool:
        """Admit a case; False when the batch is full or over its budget."""
        code = lib().xcal_batch_add(self.h, case.h, int(charge_bytes))
        if code == _abi.XCAL_ERR_BUSY:
            return False
        check(code, self.ctx.h)
        self.cases.append(case)
        return True

    def remove(self, case: Case) -> None:
        check(lib().xcal_batch_remove(self.h, case.h), self.ctx.h)
        self.cases.remove(case)

    def timings(self) -> dict:
        """Host wall time (ms) of the batch iterations so far, by phase."""
        a = np.zeros(4)
        check(lib().xcal_batch_timings(self.h, _abi.ptr(a, C.c_double)), self.ctx.h)
        return {"face_loops": a[0], "U_solves": a[1], "p_solve": a[2], "total": a[3]}

    def info(self) -> tuple[int, int, int]:
        n, used, budget = C.c_int32(), C.c_int64(), C.c_int64()
        check(lib().xcal_batch_info(self.h, C.byref(n), C.byref(used), C.byref(budget)), self.ctx.h)
        return n.value, used.value, budget.value

    def simple_iterate(self):
        """One SIMPLE iteration of every case: (residuals [n, 4], converged [n])
        in the order of ``self.cases`` before the call.  A case whose residual
        became NaN/Inf has left the batch (the others are unaffected): it is
        listed in ``self.last_diverged`` and its ``converged`` entry is
        False."""
        n = len(self.cases)
        res = np.zeros((max(n, 1), 4))
        conv = np.zeros(max(n, 1), dtype=np.int32)
        check(lib().xcal_batch_simple_iterate(self.h, _abi.ptr(res, C.c_double), _abi.ptr(conv, C.c_int32)),
              self.ctx.h)
        conv = conv[:n]
        self.last_diverged = [c for c, s in zip(self.cases, conv) if s == _abi.XCAL_ERR_DIVERGED]
        for c in self.last_diverged:
            self.cases.remove(c)
        return res[:n], conv == 1


def launch_count() -> int:
    n = C.c_int64()
    lib().xcal_get_launch_count(None, C.byref(n))
    return n.value


# ---------------------------------------------------------------------------
# run!
# ---------------------------------------------------------------------------
_CTX_CACHE: dict = {}


class VTK:
    """Output format: .vtu files (src/IOFormats/VTK/VTK_writer_3D.jl)."""


class OpenFOAM:
    """Output format: an OpenFOAM case directory (src/IOFormats/OpenFOAM/OpenFOAM_writer.jl)."""


CHECKPOINT_FIELDS = ("FIELD_U", "FIELD_P", "FIELD_MDOTF", "FIELD_NUEFF", "FIELD_GRADP", "FIELD_GRADU", "FIELD_RD",
                     "FIELD_HV", "FIELD_DIVHV", "FIELD_NUT", "FIELD_NUTF", "FIELD_UF", "FIELD_PF", "FIELD_RDF")
KOMEGA_FIELDS = ("FIELD_K", "FIELD_OMEGA")  # checkpointed for RANS{KOmega} cases


def boundary_average(patch: str, field, fieldBCs, config=None, *, mesh: Mesh3, time: float = 0.0):
    """boundary_average(patch, field, fieldBCs, config; time)
    (Postprocess_functions.jl:157-185): the mean over the patch's faces of the
    field's boundary face values (the boundary interpolation of its BC on
    that patch: Dirichlet and vector Wall the value; Zerogradient,
    Extrapolated, scalar Wall and scalar Symmetry the owner cell's value;
    vector Symmetry the cell value less its normal part; Empty zero),
    summed face by face in patch order and divided by the face count.
    ``field``: [n] (scalar) or [3, n] (vector); returns a float or a [3]
    array."""
    rng = mesh.patch_range(patch)
    bc = next((b for b in fieldBCs if b.name == patch), None)
    if bc is None:
        raise KeyError(f'no boundary condition for patch "{patch}"')
    f = np.asarray(field, dtype=np.float64)
    vector = f.ndim == 2
    ids = np.arange(rng.start, rng.stop)
    cells = np.asarray(mesh.boundary_cellsID)[ids]
    cell_vals = f[:, cells].T if vector else f[cells]
    k = bc.kind
    if k == _abi.BC_DIRICHLET or (k == _abi.BC_WALL and vector):
        vals = np.broadcast_to(np.asarray(bc.value, dtype=np.float64), cell_vals.shape)
    elif k == _abi.BC_DIRICHLET_FUNCTION:
        v = dirichlet_function_values(mesh, bc, 3 if vector else 1, time)
        vals = v.reshape(-1, 3) if vector else v.reshape(-1)
    elif k in (_abi.BC_ZEROGRADIENT, _abi.BC_EXTRAPOLATED, _abi.BC_WALL) or (k == _abi.BC_SYMMETRY and not vector):
        vals = cell_vals
    elif k == _abi.BC_SYMMETRY:
        n = np.asarray(mesh.face_normal)[ids]
        dn = np.sum(cell_vals * n, axis=1, keepdims=True)
        vals = cell_vals - dn * n
    elif k == _abi.BC_EMPTY:
        vals = np.zeros_like(cell_vals)
    else:
        raise NotImplementedError(f"boundary_average: boundary kind {k} (Neumann, periodic) is not supported")
    total = np.cumsum(vals, axis=0)[-1]  # sequential, as `sum += faceField[fID]`
    return total / len(rng) if vector else float(total / len(rng))


def save_checkpoint(state: dict, path: str) -> None:
    """Write a Case.checkpoint() to ``path`` (numpy .npz, exact doubles)."""
    np.savez(path, **state)


def load_checkpoint(path: str) -> dict:
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def _output_fields(case, model, transient_les: bool):
    """The fields save_output writes per turbulence model (isothermal):
    U, p; then k, omega, nut (RANS_kOmega.jl:236-246), with y (KOmegaSST,
    RANS_kOmegaSST.jl:323-336), with kl and y (KOmegaLKE,
    RANS_kOmegaLKE.jl:478-489); k, nut (LES_KEquation.jl:198-207); nut for
    transient Smagorinsky."""
    fields = [("U", case.get_field(_abi.FIELD_U)), ("p", case.get_field(_abi.FIELD_P))]
    t = model.turbulence
    names = []
    if isinstance(t, RANS) and t.model in (KOmega, KOmegaSST, KOmegaLKE):
        names = ["k", "omega"] + (["kl"] if t.model is KOmegaLKE else []) + ["nut"]
        names += ["y"] if t.model in (KOmegaSST, KOmegaLKE) else []
    elif isinstance(t, LES) and t.model is KEquation:
        names = ["k", "nut"]
    elif transient_les:
        names = ["nut"]
    ids = {"k": _abi.FIELD_K, "omega": _abi.FIELD_OMEGA, "kl": _abi.FIELD_KL, "nut": _abi.FIELD_NUT,
           "y": _abi.FIELD_WALLDIST}
    fields += [(n, case.get_field(ids[n])) for n in names]
    return fields


def run_(model: Physics, config: Configuration, pref=None, ncorrectors: int = 0, inner_loops=None, output=None,
         output_dir: str | None = None):
    """run! (Solvers_3_solver_dispatch.jl:120,225): SIMPLE for Steady, PISO
    for Transient.  Returns the residual histories (Ux, Uy, Uz, p) and writes
    the final fields back into ``model.momentum``.

    Results are written as the reference writes them (Solvers_1_SIMPLE.jl:
    235-257, Solvers_2_PISO.jl:205): every ``runtime.write_interval``
    iterations and, for SIMPLE, at convergence; nothing when write_interval
    is negative.  ``output``: VTK() (default) or OpenFOAM(); files go to
    ``output_dir`` (default: the working directory), written on a
    background thread while the solve continues."""
    if ncorrectors != 0 and isinstance(model.time, Transient):
        raise NotImplementedError("non-orthogonal correctors are implemented for SIMPLE (steady) runs")
    backend = config.hardware.backend
    if not isinstance(backend, B200Backend):
        raise TypeError("Hardware.backend must be B200Backend() for this implementation")
    dev = backend.device
    if dev not in _CTX_CACHE:
        _CTX_CACHE[dev] = Context(dev)
    ctx = _CTX_CACHE[dev]
    cfg, keep = build_config(model, config, pref, inner_loops, ncorrectors)
    dmesh = DeviceMesh(ctx, model.domain)
    case = Case(dmesh, cfg)
    wi = int(config.runtime.write_interval)
    transient = isinstance(model.time, Transient)
    writer = aw = None
    if wi > 0 or (wi == 0 and not transient):
        import os
        from .writers import AsyncWriter, FOAMWriter, VTKWriter2D, VTKWriter3D
        pm = model.domain.polymesh
        out_dir = output_dir or os.getcwd()
        if pm is None and getattr(model.domain, "cell_nodes", None) is not None:
            if isinstance(output, OpenFOAM):  # initialise_writer(::OpenFOAM, mesh) takes a Mesh3 only
                raise ValueError("OpenFOAM output needs a 3D mesh; this 2D mesh writes VTK")
            writer = VTKWriter2D(model.domain.points, model.domain.cell_nodes)
        elif pm is None:
            raise ValueError("writing results needs the mesh's nodes and faces (a mesh from build_mesh3, "
                             "FOAM3D_mesh, UNV3D_mesh or UNV2D_mesh)")
        else:
            writer = (FOAMWriter(pm, out_dir, config.boundaries) if isinstance(output, OpenFOAM)
                      else VTKWriter3D(pm))
        aw = AsyncWriter()

    def write(k):
        fields = _output_fields(case, model, transient and isinstance(model.turbulence, LES))
        if isinstance(writer, FOAMWriter):
            tdir = ("%.8f" % (k * config.runtime.time_step)) if transient else "%d" % k
            aw.submit(writer.write, tdir, fields)
        else:
            ext = "vtk" if isinstance(writer, VTKWriter2D) else "vtu"
            name = ("time_%d." if transient else "iteration_%d.") % k + ext
            aw.submit(writer.write, os.path.join(out_dir, name), fields)

    try:
        case.set_field(_abi.FIELD_U, model.momentum.U)
        case.set_field(_abi.FIELD_P, model.momentum.p)
        if hasattr(model.turbulence, "k"):
            case.set_field(_abi.FIELD_K, model.turbulence.k)
            if hasattr(model.turbulence, "omega"):
                case.set_field(_abi.FIELD_OMEGA, model.turbulence.omega)
            if hasattr(model.turbulence, "kl"):
                case.set_field(_abi.FIELD_KL, model.turbulence.kl)
            case.set_field(_abi.FIELD_NUT, model.turbulence.nut)
        n = config.runtime.iterations
        step = wi if wi > 0 else n
        hist, done = [], 0
        while done < n:
            k = min(step, n - done)
            if transient:
                r, _ = case.piso_step(k)
                conv = False
            else:
                r, conv = case.simple_iterate(k)
            hist.append(r)
            done += len(r)
            if conv and writer is not None:
                write(done)
                break
            if conv:
                break
            if wi > 0 and done % wi == 0:
                write(done)
        res = np.concatenate(hist, axis=0) if hist else np.zeros((0, 4))
        hits = case.solve_report()["itmax_hits"]
        if hits:
            # solve_system! warns for every solve that stopped at itmax
            # (Solve_1_api.jl:302); the run carries on, as there
            import warnings
            warnings.warn(f"Maximum number of iterations reached! ({hits} Krylov solves stopped at itmax)",
                          RuntimeWarning, stacklevel=2)
        model.momentum.U[:] = case.get_field(_abi.FIELD_U)
        model.momentum.p[:] = case.get_field(_abi.FIELD_P)
        if isinstance(model.turbulence, LES) or hasattr(model.turbulence, "k"):
            model.nut[:] = case.get_field(_abi.FIELD_NUT)
        if hasattr(model.turbulence, "k"):
            model.turbulence.k[:] = case.get_field(_abi.FIELD_K)
            if hasattr(model.turbulence, "omega"):
                model.turbulence.omega[:] = case.get_field(_abi.FIELD_OMEGA)
            if hasattr(model.turbulence, "kl"):
                model.turbulence.kl[:] = case.get_field(_abi.FIELD_KL)
            if hasattr(model.turbulence, "y"):
                model.turbulence.y[:] = case.get_field(_abi.FIELD_WALLDIST)
    finally:
        if aw is not None:
            aw.close()
        case.close()
        dmesh.close()
    return {"Ux": res[:, 0], "Uy": res[:, 1], "Uz": res[:, 2], "p": res[:, 3]}
