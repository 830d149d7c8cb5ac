"""The reference's equation DSL, carried across the C boundary as a term list.

    eqn = (Time[Euler](T) + Divergence[Upwind](mdotf, T) - Laplacian[Linear](kappa, T)
           + Si(d, T) == Source(s)) >> ScalarEquation(T, bcs)

follows ModelFramework_0_types.jl:18-100 and ModelFramework_1_operations.jl:
3-63: an operator has a flux, the field it acts on, a sign and a type;
``a + b`` collects operators in order, ``a - b`` collects them and sets the
sign of ``b`` to -1 (it is set, not flipped), ``-a`` sets the sign of ``a``;
sources combine the same way; ``terms == sources`` makes a Model, and
``model >> ScalarEquation(phi, bcs)`` stands for ``model → ScalarEquation``
(Python has no ``→``).  A flux is a per-face array (Divergence, Laplacian),
a per-cell array (Time, Si) or a number (a ConstantScalar).

On the device the equation is an :class:`Equation` (xcal_equation_*):
``discretise``, ``apply_boundary_conditions``, ``system`` and ``solve``
mirror discretise!, apply_boundary_conditions! and solve_system!.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, replace

import numpy as np

from . import _abi
from . import api as A
from ._lib import check, lib


@dataclass
class Operator:
    """Operator{F,P,S,T}: flux, the field it acts on (phi), sign, type."""
    op: int
    scheme: int
    flux: object
    phi: object
    sign: float = 1.0

    def __add__(self, other):
        return _Terms([self]) + other

    def __sub__(self, other):
        return _Terms([self]) - other

    def __neg__(self):
        return _Terms([replace(self, sign=-1.0)])

    def __eq__(self, sources):  # the DSL's `==`: an equation, not a comparison
        return _Terms([self]) == sources

    __hash__ = None


class _Terms(list):
    def __add__(self, other: Operator):
        return _Terms(list(self) + [other])

    def __sub__(self, other: Operator):
        return _Terms(list(self) + [replace(other, sign=-1.0)])

    def __eq__(self, sources):
        src = list(sources) if isinstance(sources, _Sources) else [sources]
        return Model(list(self), src)

    __hash__ = None


def _scheme_op(op, scheme_of):
    class _Op:
        def __class_getitem__(cls, scheme):
            code = scheme_of(scheme)

            def make(*args):
                if len(args) == 1 and op == _abi.OP_TIME:  # Time{T}(phi): flux ConstantScalar(1)
                    return Operator(op, code, 1.0, args[0])
                flux, phi = args
                return Operator(op, code, flux, phi)
            return make
    return _Op


def _time_code(s):
    return _abi.TIME_EULER if A._kind(s) is A.Euler else _abi.TIME_STEADY


def _div_code(s):
    k = A._kind(s)
    return {A.Linear: _abi.DIV_LINEAR, A.Upwind: _abi.DIV_UPWIND, A.LUST: _abi.DIV_LUST}[k]


def _lap_code(s):
    if A._kind(s) is not A.Linear:
        raise NotImplementedError("Laplacian{Linear} is the Laplacian on this path")
    return 0


Time = _scheme_op(_abi.OP_TIME, _time_code)
Divergence = _scheme_op(_abi.OP_DIVERGENCE, _div_code)
Laplacian = _scheme_op(_abi.OP_LAPLACIAN, _lap_code)


def Si(flux, phi) -> Operator:
    """Implicit source Si(flux, phi): flux * V on the diagonal."""
    return Operator(_abi.OP_SI, 0, flux, phi)


@dataclass
class Src:
    """Src{F,S}: a source field (per cell, or a number) and its sign."""
    field: object
    sign: float = 1.0

    def __add__(self, other):
        return _Sources([self]) + other

    def __sub__(self, other):
        return _Sources([self]) - other

    def __neg__(self):
        return _Sources([replace(self, sign=-1.0)])


class _Sources(list):
    def __add__(self, other: Src):
        return _Sources(list(self) + [other])

    def __sub__(self, other: Src):
        return _Sources(list(self) + [replace(other, sign=-1.0)])


def Source(field) -> Src:
    return Src(field, 1.0)


@dataclass
class Model:
    """Model{TN,SN}: the terms and sources of an equation."""
    terms: list
    sources: list

    def __rshift__(self, eqn: "ScalarEquation") -> "ModelEquation":
        return ModelEquation(self, eqn.phi, list(eqn.bcs))


@dataclass
class ScalarEquation:
    """The target of ``→``: the unknown (n_cells values) and its boundary
    conditions (Dirichlet, Neumann, Zerogradient, Extrapolated, Wall,
    Symmetry, Empty, DirichletFunction)."""
    phi: np.ndarray
    bcs: list


@dataclass
class ModelEquation:
    model: Model
    phi: np.ndarray
    bcs: list


class Equation:
    """A ModelEquation assembled and solved by libxcal_b200 on a case's mesh."""

    def __init__(self, case: A.Case, eqn: ModelEquation):
        self.case = case
        mesh = case.mesh
        self._keep = []
        n_t, n_s = len(eqn.model.terms), len(eqn.model.sources)
        terms = (_abi.TermDesc * n_t)()
        for k, t in enumerate(eqn.model.terms):
            face = t.op in (_abi.OP_DIVERGENCE, _abi.OP_LAPLACIAN)
            terms[k].op, terms[k].scheme, terms[k].sign = t.op, t.scheme, float(t.sign)
            self._flux(terms[k], t.flux, mesh.n_faces if face else mesh.n_cells, "flux")
        srcs = (_abi.SourceDesc * max(1, n_s))()
        for k, s in enumerate(eqn.model.sources):
            srcs[k].sign = float(s.sign)
            self._flux(srcs[k], s.field, mesh.n_cells, "field")
        bcs = A._bc_array(mesh, eqn.bcs, 1, self._keep)
        h = C.c_void_p()
        check(lib().xcal_equation_create(case.h, n_t, terms, n_s, srcs, len(eqn.bcs), bcs, C.byref(h)),
              case.dmesh.ctx.h)
        self.h = h
        self.n = mesh.n_cells

    def _flux(self, desc, v, n, name):
        if np.isscalar(v):
            desc.value = float(v)
            setattr(desc, name, None)
            return
        a = np.ascontiguousarray(v, dtype=np.float64).ravel()
        if a.size != n:
            raise ValueError(f"a flux / source array has {a.size} values, {n} expected")
        self._keep.append(a)
        setattr(desc, name, _abi.ptr(a, C.c_double))

    def _chk(self, code):
        check(code, self.case.dmesh.ctx.h)

    def _live(self):
        if not getattr(self, "h", None) or not getattr(self.case, "h", None):
            raise RuntimeError("the equation or its case has been closed")

    def close(self):
        if getattr(self, "h", None):
            lib().xcal_equation_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def discretise(self, prev=None, dt: float = 0.0):
        """discretise!(eqn, prev, config): prev = the previous values read
        by Time{Euler} (None without one), dt its time step."""
        self._live()
        p = None
        if prev is not None:
            p = np.ascontiguousarray(prev, dtype=np.float64)
            self._keep.append(p)
        self._chk(lib().xcal_equation_discretise(self.h, _abi.ptr(p, C.c_double) if p is not None else None,
                                                 float(dt)))

    def apply_boundary_conditions(self, phi=None):
        """apply_boundary_conditions!(eqn, BCs) with the field's current
        values (read by Extrapolated boundaries)."""
        self._live()
        p = None if phi is None else np.ascontiguousarray(phi, dtype=np.float64)
        self._chk(lib().xcal_equation_apply_bcs(self.h, _abi.ptr(p, C.c_double) if p is not None else None))

    def system(self):
        """(rowptr, colval, nzval, b) in the original numbering."""
        self._live()
        nnz = C.c_int64()
        self._chk(lib().xcal_equation_nnz(self.h, C.byref(nnz)))
        rp = np.empty(self.n + 1, dtype=np.int32)
        cv = np.empty(nnz.value, dtype=np.int32)
        nz = np.empty(nnz.value)
        b = np.empty(self.n)
        self._chk(lib().xcal_equation_get_system(self.h, _abi.ptr(rp, C.c_int32), _abi.ptr(cv, C.c_int32),
                                                 _abi.ptr(nz, C.c_double), _abi.ptr(b, C.c_double)))
        return rp, cv, nz, b

    def solve(self, setup: A.SolverSetup, phi):
        """solve_system! in FP64 from the initial guess phi: (solution,
        scaled residual, Krylov iterations)."""
        self._live()
        x = np.array(phi, dtype=np.float64, copy=True)
        res, its = C.c_double(), C.c_int32()
        desc = A._solver_desc(setup)
        self._chk(lib().xcal_equation_solve(self.h, C.byref(desc), _abi.ptr(x, C.c_double), C.byref(res),
                                            C.byref(its)))
        return x, res.value, its.value
