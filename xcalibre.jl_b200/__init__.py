"""xcalibre.jl_b200 -- sm_100a implementation of XCALibre.jl's finite-volume
hot path behind a C ABI (libxcal_b200.so), with a host-side mirror of the
reference's user API for that path.

The directory name contains a dot, so load it with ``importlib`` (see
``__graft_entry__.load_package``); it is registered as ``xcalibre_b200``.
"""
from . import _abi, api, cases
from .api import (B200Backend, Bicgstab, Case, CellBased, Cg, Configuration, Context, DeviceMesh, DILU, Dirichlet, Midpoint,
                  DirichletFunction, Empty, Energy, Euler, Extrapolated, Fluid, Gauss, Hardware, Incompressible,
                  Isothermal, Jacobi, LES, LUST, Laminar, Linear, Neumann, Physics, RANS, Runtime, Schemes,
                  Smagorinsky, SolverSetup, Steady, SteadyState, Symmetry, Transient, Upwind, Wall, Zerogradient,
                  assign, build_config, construct_periodic, initialise_, launch_count, run_, Batch,
                  footprint_estimate, VTK, OpenFOAM, save_checkpoint, load_checkpoint, boundary_average, JacobiSmoother,
                  KOmega, KOmegaSST, KOmegaLKE, OmegaWallFunction, KWallFunction, NutWallFunction, KEquation)
from . import dsl
from .dsl import Divergence, Equation, Laplacian, ScalarEquation, Si, Source, Time
from .foam import Mesh3, build_mesh3
from .foamio import FOAM3D_mesh, read_polymesh, write_polymesh
from .unv import UNV2D_mesh, UNV3D_mesh
from .meshgen import (PolyMesh, box_polymesh, cavity_polymesh, channel_polymesh, flatplate_polymesh,
                      periodic_box_polymesh)

__all__ = [n for n in dir() if not n.startswith("_")] + ["_abi"]
