/*
 * xcal_b200.h -- C ABI of libxcal_b200.so, the sm_100a implementation of the
 * XCALibre.jl finite-volume hot path (assembly -> CSR, Gauss gradients, face
 * interpolation, CG/BiCGSTAB with Jacobi/DILU, SIMPLE/PISO corrections).
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and returns
 * an int32_t status (XCAL_OK == 0, negative on error; xcal_last_error() gives the
 * message).  Indices in this ABI are 0-based; the Julia side subtracts 1.
 *
 * Each declaration names the reference function it replaces (paths are relative
 * to the XCALibre.jl project root).
 */
#ifndef XCAL_B200_H
#define XCAL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
enum {
    XCAL_OK = 0,
    XCAL_ERR_INVALID = -1,        /* bad argument, mesh or config            */
    XCAL_ERR_CUDA = -2,           /* CUDA runtime error                      */
    XCAL_ERR_OOM = -3,            /* device allocation failed                */
    XCAL_ERR_NOT_CONVERGED = -4,  /* outer loop ended without convergence   */
    XCAL_ERR_DIVERGED = -5,       /* NaN/Inf seen in a residual             */
    XCAL_ERR_TIMEOUT = -6,        /* a bounded device wait gave up          */
    XCAL_ERR_UNSUPPORTED = -7,    /* option outside the implemented path    */
    XCAL_ERR_BUSY = -8            /* batch full or device-memory budget hit */
};

/* ---- enumerations mirroring the reference's dispatch types ------------- */
/* boundary conditions: src/Discretise/boundary_conditions/ *.jl           */
enum {
    XCAL_BC_DIRICHLET = 1,          /* dirichlet.jl                          */
    XCAL_BC_DIRICHLET_FUNCTION = 2, /* dirichletFunction.jl (values per face)*/
    XCAL_BC_WALL = 3,               /* wall.jl                               */
    XCAL_BC_ZEROGRADIENT = 4,       /* zerogradient.jl                       */
    XCAL_BC_EXTRAPOLATED = 5,       /* extrapolated.jl                       */
    XCAL_BC_EMPTY = 6,              /* empty.jl                              */
    XCAL_BC_SYMMETRY = 7,           /* symmetry.jl                           */
    XCAL_BC_NEUMANN = 8,            /* neumann.jl (scalar fields)            */
    XCAL_BC_PERIODIC = 9,           /* periodic.jl `Periodic` (shadow side)  */
    XCAL_BC_PERIODIC_PARENT = 10,   /* periodic.jl `PeriodicParent`          */
    XCAL_BC_OMEGA_WALL = 11,        /* OmegaWallFunction (Discretise_0_types.jl:
                                       83-113; constraint RANS_functions.jl:
                                       376-429): constants in xcal_bc.wall  */
    XCAL_BC_K_WALL = 12,            /* KWallFunction (production, RANS_functions.jl:
                                       66-117)                               */
    XCAL_BC_NUT_WALL = 13           /* NutWallFunction (nutf, :119-172)      */
};
/* Time{T}: src/Discretise/Discretise_1_schemes.jl:12-45 */
enum { XCAL_TIME_STEADY = 0, XCAL_TIME_EULER = 1 };
/* Divergence{T}: src/Discretise/Discretise_1_schemes.jl:114-180 */
enum { XCAL_DIV_LINEAR = 0, XCAL_DIV_UPWIND = 1, XCAL_DIV_LUST = 2 };
/* gradient schemes: Gauss (Calculate_1_green_gauss.jl) and Midpoint
 * (Calculate_0_gradient.jl:170-262: midpoint face values, Green-Gauss, then
 * two rounds of gradient-corrected face values and Green-Gauss) */
enum { XCAL_GRAD_GAUSS = 0, XCAL_GRAD_MIDPOINT = 1 };
/* gradient limiters: none, or CellBased (Calculate_0_gradient_cell_limiter.jl,
 * Barth-Jespersen, strength level); p_schemes: after every grad p, U_schemes:
 * after grad U in the turbulence update, per component (nut after it) */
/* CellBased(level) (Calculate_0_gradient_cell_limiter.jl); FaceBased
 * (Calculate_0_gradient_face_limiter.jl: per cell the minimum over its
 * internal faces, no level); MFaceBased
 * (Calculate_0_gradient_mface_limiter.jl: each internal face corrects both
 * cells' gradients in turn; the library applies a cell's faces in ascending
 * face order, the reference run on one thread) */
enum { XCAL_LIMITER_NONE = 0, XCAL_LIMITER_CELL = 1, XCAL_LIMITER_FACE = 2, XCAL_LIMITER_MFACE = 3 };
/* Krylov solver: src/Solve/Solve_1_Krylov_solvers.jl:6-15 */
enum { XCAL_SOLVER_CG = 0, XCAL_SOLVER_BICGSTAB = 1 };
/* preconditioner: src/Solve/Preconditioners/preconditioners_0_types.jl */
enum { XCAL_PRECOND_NONE = 0, XCAL_PRECOND_JACOBI = 1, XCAL_PRECOND_DILU = 2 };
/* turbulence: RANS{Laminar} / LES{Smagorinsky} / RANS{KOmega} */
enum {
    XCAL_TURB_LAMINAR = 0,
    XCAL_TURB_SMAGORINSKY = 1,
    XCAL_TURB_KOMEGA = 2,
    XCAL_TURB_KOMEGA_SST = 3,
    XCAL_TURB_KEQUATION = 4,  /* LES{KEquation} (LES_KEquation.jl) */
    XCAL_TURB_KOMEGA_LKE = 5  /* RANS{KOmegaLKE} (RANS_kOmegaLKE.jl): k, omega
                                 and the laminar kinetic energy kl */
};
/* arithmetic of the Krylov inner iterations */
enum { XCAL_PREC_FP64 = 0, XCAL_PREC_MIXED = 1 };
/* pressure-velocity algorithm: run! dispatch, src/Solvers/Solvers_3_solver_dispatch.jl:120,225 */
enum { XCAL_ALGO_SIMPLE = 0, XCAL_ALGO_PISO = 1 };
/* equations (k, omega: RANS{KOmega} transport equations) */
enum { XCAL_EQN_U = 0, XCAL_EQN_P = 1, XCAL_EQN_K = 2, XCAL_EQN_OMEGA = 3, XCAL_EQN_WALLDIST = 4,
       XCAL_EQN_KL = 5 /* RANS{KOmegaLKE} laminar kinetic energy */ };

/* field identifiers for xcal_case_get_field / xcal_case_set_field.
 * Cell fields hold n_cells values per component, face fields n_faces; vector
 * fields are stored component-major (all x, then all y, then all z), tensor
 * fields in the order xx,xy,xz,yx,yy,yz,zx,zy,zz (res[i,j] = d u_i / d x_j). */
enum {
    XCAL_FIELD_U = 0,      /* VectorField U (3 x n_cells)                   */
    XCAL_FIELD_P = 1,      /* ScalarField p                                 */
    XCAL_FIELD_MDOTF = 2,  /* FaceScalarField mdotf                         */
    XCAL_FIELD_NUEFF = 3,  /* FaceScalarField nueff                         */
    XCAL_FIELD_GRADP = 4,  /* Grad{Gauss}(p).result (3 x n_cells)           */
    XCAL_FIELD_GRADU = 5,  /* Grad{Gauss}(U).result (9 x n_cells)           */
    XCAL_FIELD_RD = 6,     /* rD (n_cells)                                  */
    XCAL_FIELD_HV = 7,     /* Hv (3 x n_cells)                              */
    XCAL_FIELD_DIVHV = 8,  /* divHv (n_cells)                               */
    XCAL_FIELD_NUT = 9,    /* nut (n_cells)                                 */
    XCAL_FIELD_NUTF = 10,  /* nutf (n_faces)                                */
    XCAL_FIELD_UF = 11,    /* Uf (3 x n_faces)                              */
    XCAL_FIELD_PF = 12,    /* pf (n_faces)                                  */
    XCAL_FIELD_RDF = 13,   /* rDf (n_faces)                                 */
    XCAL_FIELD_DELTA = 14, /* LES filter: (C*Delta)^2 (Smagorinsky), Delta
                              (KEquation) (n_cells)                     */
    XCAL_FIELD_K = 15,     /* k: RANS{KOmega*}, LES{KEquation} (n_cells)    */
    XCAL_FIELD_OMEGA = 16, /* RANS{KOmega*} omega (n_cells)                 */
    XCAL_FIELD_WALLDIST = 17, /* RANS{KOmegaSST, KOmegaLKE} wall distance y */
    XCAL_FIELD_PK = 18,    /* the k equation's Source (n_cells)             */
    XCAL_FIELD_DK = 19,    /* the k equation's Si coefficient (n_cells)     */
    XCAL_FIELD_DW = 20,    /* omega's Si coefficient (k-omega), the k
                              equation's second Si coefficient (KEquation) */
    XCAL_FIELD_KL = 21,    /* RANS{KOmegaLKE} laminar kinetic energy kl     */
    XCAL_FIELD_GAMMA = 22, /* RANS{KOmegaLKE} intermittency trigger gamma   */
    XCAL_FIELD_COUNT = 23
};

/* ---- mesh: the Mesh3 contract (src/Mesh/Mesh_0_types.jl:28-205) ---------
 * Faces 0..n_bfaces-1 are boundary faces, patch-contiguous, with
 * face_owner[f] == face_neigh[f]; faces n_bfaces..n_faces-1 are internal.
 * cell_faces lists each cell's INTERNAL faces (owner before neighbour in
 * increasing face order, src/FoamMesh/FoamMesh_2_connect.jl:24-69) with the
 * normal sign (+1 owner, -1 neighbour) and the cell across the face.
 * Vectors are interleaved xyz (3 doubles per face/cell).                    */
typedef struct {
    int32_t n_cells;
    int32_t n_faces;
    int32_t n_bfaces;
    const int32_t* face_owner;        /* [n_faces]  ownerCells[1]            */
    const int32_t* face_neigh;        /* [n_faces]  ownerCells[2]            */
    const double* face_centre;        /* [3*n_faces]                         */
    const double* face_normal;        /* [3*n_faces]                         */
    const double* face_e;             /* [3*n_faces]                         */
    const double* face_area;          /* [n_faces]                           */
    const double* face_delta;         /* [n_faces]                           */
    const double* face_weight;        /* [n_faces]                           */
    const double* cell_centre;        /* [3*n_cells]                         */
    const double* cell_volume;        /* [n_cells]                           */
    const int32_t* cell_faces_offset; /* [n_cells+1] (faces_range)           */
    const int32_t* cell_faces;        /* [2*n_ifaces]                        */
    const int32_t* cell_nsign;        /* [2*n_ifaces]                        */
    const int32_t* cell_neighbours;   /* [2*n_ifaces]                        */
    const int32_t* boundary_cellsID;  /* [n_bfaces]                          */
    int32_t n_patches;
    const int32_t* patch_start;       /* [n_patches] first face id           */
    const int32_t* patch_count;       /* [n_patches]                         */
    int32_t dim;                      /* 2: a Mesh2 (UNV2D_mesh; Courant cell
                                         size sqrt(V), Solvers_0_functions.jl:
                                         277-285); 0 or 3: a Mesh3           */
} xcal_mesh_desc;

/* ---- boundary condition (one per patch per field) ----------------------
 * Mirrors the functor structs in src/Discretise/boundary_conditions/
 * after `assign` (src/Discretise/Discretise_4_assign_boundaries.jl:5).      */
typedef struct {
    int32_t type;               /* XCAL_BC_*                                 */
    int32_t patch;              /* patch index into the mesh's patch list   */
    double value[3];            /* scalar in value[0], vector in value[0..2]*/
    /* DirichletFunction: values of f(face.centre, time, i) for the patch's
     * faces, evaluated by the caller (components interleaved for vectors). */
    const double* face_values;
    /* Periodic / PeriodicParent (construct_periodic, periodic.jl:95-217)  */
    const int32_t* face_map;    /* [patch_count] partner face ids           */
    double distance[3];         /* LinearTransform.distance                 */
    int32_t partner_patch;
    /* wall functions: kappa, beta1, cmu^0.25, yPlusLam =
     * y_plus_laminar(E, kappa) (RANS_functions.jl:42-49) and E, evaluated by
     * the caller */
    double wall[5];
} xcal_bc;

/* SolverSetup (src/Solve/Solve_1_api.jl:8-83) */
typedef struct {
    int32_t solver;             /* XCAL_SOLVER_*                             */
    int32_t precond;            /* XCAL_PRECOND_*                            */
    double convergence;
    double relax;
    double atol;
    double rtol;
    int32_t itmax;
    int32_t smoother_loops;     /* JacobiSmoother(loops, omega): weighted
                                   Jacobi sweeps on the field before each
                                   Krylov solve (Smoothers_jacobi.jl:56-132,
                                   Solve_1_api.jl:284); 0 = no smoother      */
    double smoother_omega;
} xcal_solver_setup;

/* Schemes (src/Solve/Solve_1_api.jl:205-211); the Laplacian is always
 * Linear on this path. */
typedef struct {
    int32_t time;               /* XCAL_TIME_*                               */
    int32_t divergence;         /* XCAL_DIV_*                                */
    int32_t gradient;           /* XCAL_GRAD_* (p: grad p; U: grad U)       */
    int32_t limiter;            /* XCAL_LIMITER_*                            */
    double limiter_level;       /* CellBased(level), 0..1                    */
} xcal_schemes;

/* Configuration + Physics (src/Simulate/Simulate_0_types.jl:32-74,
 * src/ModelPhysics/0_type_definition.jl:196-229) reduced to what the hot
 * path reads. */
typedef struct {
    int32_t algorithm;          /* XCAL_ALGO_SIMPLE / XCAL_ALGO_PISO         */
    int32_t turbulence;         /* XCAL_TURB_*                               */
    double nu;                  /* Fluid{Incompressible}(nu)                 */
    double smagorinsky_C;       /* LES{Smagorinsky}(C)                       */
    /* LES filter width Delta = C (V / les_delta_distance)^les_delta_power,
     * from delta_scaling(mesh, BCs) (LES_functions.jl:33-56): (the distance
     * between the Empty patches, 0.5) for a 2D slab, else (1, 1/3).  Power 0
     * = not given: the library takes the first Empty patch of the U BCs and
     * the box of the boundary-face centres (the reference's box spans the
     * boundary faces' nodes; the two agree when the patch normal is
     * axis-aligned). */
    double les_delta_distance;
    double les_delta_power;
    xcal_schemes U_schemes;
    xcal_schemes p_schemes;
    xcal_solver_setup U_solver;
    xcal_solver_setup p_solver;
    int32_t iterations;         /* Runtime.iterations                        */
    double dt;                  /* Runtime.dt (time step; 1 for steady)      */
    int32_t has_pref;           /* run!(...; pref) given                     */
    double pref;
    int32_t inner_loops;        /* PISO correctors (run!(...; inner_loops))  */
    int32_t ncorrectors;        /* SIMPLE non-orthogonal correctors
                                   (run!(...; ncorrectors),
                                   Solvers_1_SIMPLE.jl:196-206); PISO: 0  */
    int32_t precision;          /* XCAL_PREC_*                               */
    double inner_rtol;          /* mixed: relative tolerance of each FP32
                                   inner solve (0 = default 1e-3)            */
    int32_t n_bc_U, n_bc_p, n_bc_nut;
    const xcal_bc* bc_U;
    const xcal_bc* bc_p;
    const xcal_bc* bc_nut;
    /* RANS{KOmega} (RANS_kOmega.jl:29-52): coefficients beta_star (beta+),
     * alpha1, beta1, sigma_k, sigma_omega; the k and omega equations' schemes
     * (time, divergence) and solver setups (omega is solved with k's
     * preconditioner type, :84-85); their boundary conditions */
    double kw_beta_star, kw_alpha1, kw_beta1, kw_sigma_k, kw_sigma_omega;
    xcal_schemes k_schemes;
    xcal_schemes omega_schemes;
    xcal_solver_setup k_solver;
    xcal_solver_setup omega_solver;
    int32_t n_bc_k, n_bc_omega;
    const xcal_bc* bc_k;
    const xcal_bc* bc_omega;
    /* RANS{KOmegaSST} (RANS_kOmegaSST.jl:57-79): beta+, alpha1, beta1,
     * sigma_k1, sigma_omega1 in kw_*, and beta2, sigma_k2, sigma_omega2
     * here; grad k uses k_schemes.gradient, grad omega p_schemes.gradient
     * (:146-147); the wall distance (wall_distance!,
     * Calculate_4_wall_distance.jl:4-78): its solver, gradient scheme and
     * BCs (Dirichlet 0 on the walls, Empty, Extrapolated elsewhere) */
    double sst_beta2, sst_sigma_k2, sst_sigma_omega2;
    xcal_schemes y_schemes;
    xcal_solver_setup y_solver;
    int32_t n_bc_y;
    const xcal_bc* bc_y;
    /* LES{KEquation}(; ck, ce) (LES_KEquation.jl:35-39): the subgrid k
     * equation Time + Div(mdotf) - Lap(nu + nut_f) + Si(ce sqrt(k) / Delta)
     * + Si(2/3 tr grad U) == Source(2 nut grad U : dev(S)), solved with
     * k_schemes / k_solver / bc_k, then nut = ck Delta sqrt(k) with Delta =
     * (V / les_delta_distance)^les_delta_power (:80-186) */
    double keq_ck, keq_ce;
    /* RANS{KOmegaLKE}(; Tu, walls) (RANS_kOmegaLKE.jl:60-100): the
     * freestream turbulence intensity Tu (eta = 0.02974 tanh(59.79 Tu^1.191
     * + 1.65e-13); the other coefficients are the model's constants); k and
     * omega use k_* / omega_* (each equation its own preconditioner), the
     * laminar kinetic energy kl the fields below, the wall distance the y_*
     * fields (Dirichlet 0 on the walls) */
    double lke_Tu;
    xcal_schemes kl_schemes;
    xcal_solver_setup kl_solver;
    int32_t n_bc_kl;
    const xcal_bc* bc_kl;
} xcal_config;

/* ---- polyMesh input of the mesh importer --------------------------------
 * The arrays an OpenFOAM constant/polyMesh directory holds (0-based), as read
 * by read_FOAM3D (src/FoamMesh/FoamMesh_1_read.jl:1-23): internal faces
 * first, then each patch's faces in patch order. */
typedef struct {
    int32_t n_points;
    const double* points;         /* [3*n_points]                          */
    int32_t n_faces;
    const int32_t* face_offsets;  /* [n_faces+1] into face_nodes           */
    const int32_t* face_nodes;    /* [face_offsets[n_faces]]               */
    const int32_t* owner;         /* [n_faces]                             */
    int32_t n_internal_faces;
    const int32_t* neighbour;     /* [n_internal_faces]                    */
    int32_t n_patches;
    const int32_t* patch_sizes;   /* [n_patches] nFaces per patch          */
} xcal_polymesh_desc;

/* caller-owned output buffers of the importer (same layout as
 * xcal_mesh_desc; sizes from xcal_foam_mesh_sizes) */
typedef struct {
    int32_t* face_owner;
    int32_t* face_neigh;
    double* face_centre;
    double* face_normal;
    double* face_e;
    double* face_area;
    double* face_delta;
    double* face_weight;
    double* cell_centre;
    double* cell_volume;
    int32_t* cell_faces_offset;
    int32_t* cell_faces;
    int32_t* cell_nsign;
    int32_t* cell_neighbours;
    int32_t* boundary_cellsID;
    int32_t* patch_start;
    int32_t* patch_count;
} xcal_mesh_buffers;

typedef struct xcal_ctx xcal_ctx;
typedef struct xcal_mesh xcal_mesh;
typedef struct xcal_case xcal_case;
typedef struct xcal_batch xcal_batch;

/* ---- context ------------------------------------------------------------ */
/* Hardware(backend=B200Backend()) (src/Simulate/Simulate_0_types.jl:70-74) */
int32_t xcal_ctx_create(int32_t device, xcal_ctx** out);
int32_t xcal_ctx_destroy(xcal_ctx* ctx);
/* message of the calling thread's last failed call on this context (never
 * NULL; "" when it has none).  Messages are kept per host thread, so threads
 * sharing a context never read each other's errors. */
const char* xcal_last_error(const xcal_ctx* ctx);
/* library version string */
const char* xcal_version(void);

/* ---- the library's exp / log / tanh -----------------------------------------
 * No counterpart in the reference.  The k-omega SST blending (tanh) and the
 * wall functions (log) call the library's own restatements of these
 * functions, written from +, *, / and ldexp/frexp so the device and the host
 * compute them alike (Cody-Waite reduction with a Taylor series for exp of
 * y <= 0; the atanh series for log of x > 0; tanh(x) = (1 - e^-2x) /
 * (1 + e^-2x) for x >= 0).  This evaluates those same functions, compiled
 * for the host, on n inputs: which 0 = exp, 1 = log, 2 = tanh, 3 = x^-1.3
 * (k-omega LKE's Re_upsilon^-1.30, exp(-1.3 log x)); for testing their error
 * against the C library.  Needs no device. */
int32_t xcal_det_math(int32_t which, const double* in, double* out, int64_t n);

/* ---- struct layouts, for bindings -----------------------------------------
 * No counterpart in the reference (it has no C boundary).  sizeof and the
 * field offsets of the structs above as this library was compiled, so a
 * binding's mirror (Julia structs, ctypes) can be checked against them:
 * out[0] = sizeof, out[1 + k] = offset of field k in declaration order (array
 * fields: their first element).  Returns the number of values written, or
 * XCAL_ERR_INVALID for an unknown `which` or too small a `cap`.  Needs no
 * device. */
enum {
    XCAL_LAYOUT_MESH_DESC = 0,
    XCAL_LAYOUT_BC = 1,
    XCAL_LAYOUT_SOLVER_SETUP = 2,
    XCAL_LAYOUT_SCHEMES = 3,
    XCAL_LAYOUT_CONFIG = 4,
    XCAL_LAYOUT_POLYMESH_DESC = 5,
    XCAL_LAYOUT_MESH_BUFFERS = 6,
    XCAL_LAYOUT_TERM = 7,
    XCAL_LAYOUT_SOURCE = 8
};
int32_t xcal_abi_layout(int32_t which, int64_t* out, int32_t cap);

/* ---- mesh import (host) --------------------------------------------------*/
/* FOAM3D_mesh (src/FoamMesh/FoamMesh_5_build.jl:21-27) without the file
 * parsing: sizes[0..2] = n_cells, n_faces, n_bfaces of the Mesh3 built from
 * the polyMesh.  Needs no GPU. */
int32_t xcal_foam_mesh_sizes(const xcal_polymesh_desc* pm, int32_t* sizes);
/* builds the Mesh3 contract (connectivity, boundary-first face order, fan
 * geometry, weights, deltas, volumes; FoamMesh_2_connect.jl,
 * FoamMesh_3_generate.jl, FoamMesh_4_geometry.jl, Mesh_1_functions.jl:20-51)
 * into caller buffers.  Needs no GPU. */
int32_t xcal_foam_mesh_build(const xcal_polymesh_desc* pm, const xcal_mesh_buffers* out);
/* the same Mesh3 for large meshes, with its geometry (cell centres, face fan
 * geometry, weights, deltas, volumes) computed on GPU `device` by the same
 * operations in the same order: outputs identical to xcal_foam_mesh_build.
 * The connectivity stays on the host; inputs and outputs are host arrays. */
int32_t xcal_foam_mesh_build_device(int32_t device, const xcal_polymesh_desc* pm, const xcal_mesh_buffers* out);

/* ---- mesh ----------------------------------------------------------------*/
/* adapt(backend, mesh) (docs/src/user_guide/1_preprocessing.md:88): copies
 * the Mesh3 arrays to HBM as SoA and derives the CSR-slot maps that replace
 * spindex searches (src/ModelFramework/ModelFramework_0_types.jl:246-258). */
int32_t xcal_mesh_upload(xcal_ctx* ctx, const xcal_mesh_desc* desc, xcal_mesh** out);
int32_t xcal_mesh_destroy(xcal_mesh* mesh);

/* ---- case: equations, fields, solver state -------------------------------*/
/* setup_incompressible_solvers (src/Solvers/Solvers_1_SIMPLE.jl:45-101):
 * builds U_eqn (VectorEquation) and p_eqn (ScalarEquation), their CSR
 * patterns (sparse_matrix_connectivity + periodic extend_matrix,
 * ModelFramework_0_types.jl:223-243, periodic.jl:219-254), preconditioners
 * and Krylov workspaces.  Fields start at zero (initialise! sets them). */
int32_t xcal_case_create(xcal_ctx* ctx, const xcal_mesh* mesh,
                         const xcal_config* cfg, xcal_case** out);
int32_t xcal_case_destroy(xcal_case* cs);
/* nnz of the equation's CSR (U or p) */
int32_t xcal_case_nnz(const xcal_case* cs, int32_t eqn, int64_t* nnz);
/* export the CSR pattern (0-based rowptr[n+1], colval[nnz]) */
int32_t xcal_case_csr_pattern(const xcal_case* cs, int32_t eqn,
                              int32_t* rowptr, int32_t* colval);
/* export the current matrix values and right-hand side of an equation.
 * eqn U: component 0..2 selects bx/by/bz, nzval is the A of the last
 * component whose boundary conditions were applied; component -1 returns
 * A0 (the assembled matrix before boundary conditions) with bx.  */
int32_t xcal_case_get_system(const xcal_case* cs, int32_t eqn, int32_t component,
                             double* nzval, double* b);
/* initialise! (src/Fields/Fields_0_types.jl:381-401) and field transfer */
int32_t xcal_case_set_field(xcal_case* cs, int32_t field, const double* host, int64_t count);
/* Checkpoint restore (no reference counterpart: run! always starts from U
 * and p).  After the state fields of a saved case have been set (U, p,
 * MDOTF, NUEFF, GRADP, UF, PF and the rest of the readable fields), this
 * marks the state as complete: the next iteration does not redo the run's
 * initial calculations (face velocities and mass flux from U, grad p,
 * nu_eff; Solvers_1_SIMPLE.jl:150-156), so the case continues exactly as
 * the saved one would have. */
int32_t xcal_case_mark_initialised(xcal_case* cs);
int32_t xcal_case_get_field(const xcal_case* cs, int32_t field, double* host, int64_t count);
/* replace DirichletFunction face values of BC `bc_index` of field
 * (XCAL_EQN_U or XCAL_EQN_P) -- the host-evaluated f(centre, time, i) */
int32_t xcal_case_set_bc_values(xcal_case* cs, int32_t eqn, int32_t bc_index,
                                const double* values, int64_t count);

/* ---- algorithms ------------------------------------------------------------*/
/* SIMPLE outer iterations (src/Solvers/Solvers_1_SIMPLE.jl:103-263).  The
 * first call runs the initial calculations (:150-156).  res_hist receives
 * 4 residuals (Ux, Uy, Uz, p) per iteration; *converged is set when every
 * residual fell below its SolverSetup.convergence (the loop then stops). */
int32_t xcal_simple_iterate(xcal_case* cs, int32_t n_iter, double* res_hist,
                            int32_t* n_done, int32_t* converged);
/* PISO time steps (src/Solvers/Solvers_2_PISO.jl:40-211); res_hist as above,
 * courant (may be NULL) receives max_courant_number! per step. */
int32_t xcal_piso_step(xcal_case* cs, int32_t n_steps, double* res_hist,
                       double* courant, int32_t* n_done);

/* ---- fine-grained hooks (one reference function each) -------------------*/
/* interpolate!(Uf,U) + correct_boundaries! + flux! + grad!(∇p) + update_nueff!
 * (Solvers_1_SIMPLE.jl:150-156) */
int32_t xcal_initial_calculations(xcal_case* cs);
/* discretise! (src/Discretise/Discretise_2_generated_distretisation.jl:3,89) */
int32_t xcal_discretise(xcal_case* cs, int32_t eqn);
/* update_equation! + apply_boundary_conditions! (Discretise_5_apply_bcs.jl:5)
 * for one component (U: 0..2; p: 0) */
int32_t xcal_apply_boundary_conditions(xcal_case* cs, int32_t eqn, int32_t component);
/* implicit_relaxation_diagdom! (src/Solve/Solve_1_api.jl:370-411) on U */
int32_t xcal_implicit_relaxation_diagdom(xcal_case* cs, int32_t component);
/* setReference! (src/Solve/Solve_1_api.jl:414-439) on p */
int32_t xcal_set_reference(xcal_case* cs);
/* update_preconditioner! (preconditioners_2_functions.jl:65-108) */
int32_t xcal_update_preconditioner(xcal_case* cs, int32_t eqn);
/* solve_system! (src/Solve/Solve_1_api.jl:268-307): Krylov solve warm-started
 * from the field, copy back, then residual (:441-464). */
int32_t xcal_solve_system(xcal_case* cs, int32_t eqn, int32_t component,
                          double* residual, int32_t* iterations);
/* solve_equation! (src/Solve/Solve_1_api.jl:214-266); res[3] for U, res[1] p */
int32_t xcal_solve_equation(xcal_case* cs, int32_t eqn, double* res);
/* inverse_diagonal! + interpolate!(rDf, rD) + correct_interpolation_periodic
 * + remove_pressure_source! + H! (Solvers_1_SIMPLE.jl:170-174) */
int32_t xcal_pressure_predictor(xcal_case* cs);
/* interpolate!(Uf,Hv) + correct_boundaries! + flux! + div!
 * (Solvers_1_SIMPLE.jl:177-185) */
int32_t xcal_flux_divergence(xcal_case* cs);
/* explicit_relaxation! (src/Solve/Solve_1_api.jl:317-335): p = prev + a(p-prev) */
int32_t xcal_explicit_relaxation_p(xcal_case* cs, double alpha);
/* grad!(∇p, pf, p, BCs.p) (src/Calculate/Calculate_0_gradient.jl:105-111) */
int32_t xcal_grad_p(xcal_case* cs);
/* correct_mass_flux! + correct_velocity! (Solvers_1_SIMPLE.jl:210-211) */
int32_t xcal_correct(xcal_case* cs);
/* turbulence! + update_nueff! (RANS_laminar.jl:73-79, LES_Smagorinsky.jl:105-132,
 * Solvers_0_functions.jl:5-35) */
int32_t xcal_turbulence(xcal_case* cs);
/* max_courant_number! (Solvers_0_functions.jl:253-276) */
int32_t xcal_max_courant(xcal_case* cs, double* courant);

/* ---- equations from the operator DSL ----------------------------------------
 * (Time + Divergence - Laplacian + Si == Source) -> ScalarEquation
 * (ModelFramework_0_types.jl:18-100, 135-165; ModelFramework_1_operations.jl:
 * 3-63): the terms in the order written, each with the sign the DSL gave it
 * (`-` sets -1 on the operator after it), the sources likewise.  The drivers
 * (xcal_simple_iterate, xcal_piso_step) assemble their own equations; these
 * entry points take any scalar equation of these operators on a case's mesh,
 * with its own boundary conditions, and assemble, constrain and solve it
 * with the same kernels' arithmetic. */
enum { XCAL_OP_TIME = 0, XCAL_OP_DIVERGENCE = 1, XCAL_OP_LAPLACIAN = 2, XCAL_OP_SI = 3 };
typedef struct {
    int32_t op;          /* XCAL_OP_*                                        */
    int32_t scheme;      /* Time: XCAL_TIME_*; Divergence: XCAL_DIV_*;
                            Laplacian (Linear) and Si: 0                     */
    double sign;         /* +1, or -1 where the DSL put a minus before it    */
    const double* flux;  /* Divergence, Laplacian: per face [n_faces];
                            Time, Si: per cell [n_cells]; original numbering;
                            NULL: the constant `value` (a ConstantScalar)    */
    double value;
} xcal_term;
typedef struct {         /* Source(field), Src{F,S} (ModelFramework_0_types.jl:81-93) */
    double sign;
    const double* field; /* per cell [n_cells]; NULL: the constant `value`   */
    double value;
} xcal_source;
typedef struct xcal_equation xcal_equation;
/* `terms -> ScalarEquation(phi, bcs)` on cs's mesh: the CSR pattern of
 * sparse_matrix_connectivity (ModelFramework_0_types.jl:223-243), at most 8
 * terms and 8 sources (copied; host arrays are read during the call), the
 * field's boundary conditions (no periodic pairs).  Runs on cs's stream. */
int32_t xcal_equation_create(xcal_case* cs, int32_t n_terms, const xcal_term* terms, int32_t n_sources,
                             const xcal_source* sources, int32_t n_bcs, const xcal_bc* bcs, xcal_equation** out);
/* frees the equation; it may be called after its case was destroyed (every
 * other xcal_equation_* call needs the case alive) */
int32_t xcal_equation_destroy(xcal_equation* eq);
/* discretise!(eqn, prev, config) (Discretise_2_generated_distretisation.jl:
 * 90-168): prev [n_cells] = the previous values Time{Euler} reads (NULL
 * without a Time{Euler} term), dt its time step */
int32_t xcal_equation_discretise(xcal_equation* eq, const double* prev, double dt);
/* apply_boundary_conditions!(eqn, BCs) (Discretise_5_apply_bcs.jl) for a
 * scalar field: every term's boundary functor per boundary face
 * (the boundary_conditions sources); phi [n_cells] = the field's current values
 * (Extrapolated reads them; NULL when no boundary needs them) */
int32_t xcal_equation_apply_bcs(xcal_equation* eq, const double* phi);
int32_t xcal_equation_nnz(const xcal_equation* eq, int64_t* nnz);
/* the assembled system in the original numbering, rows in the reference's
 * CSR order: rowptr [n_cells+1], colval [nnz], nzval [nnz], b [n_cells]
 * (any may be NULL) */
int32_t xcal_equation_get_system(const xcal_equation* eq, int32_t* rowptr, int32_t* colval, double* nzval,
                                 double* b);
/* update_preconditioner! + solve_system! (Solve_1_api.jl:268-307) in FP64:
 * phi [n_cells] is the initial guess and receives the solution; residual =
 * the scaled residual (:441-464), iterations = Krylov iterations (either may
 * be NULL) */
int32_t xcal_equation_solve(xcal_equation* eq, const xcal_solver_setup* setup, double* phi, double* residual,
                            int32_t* iterations);

/* ---- allocation-free residual ---------------------------------------------
 * No counterpart in the reference: an extra entry point for callers that
 * cannot allocate device memory (inside CUDA graph capture, under a fixed
 * memory budget or a caller-managed pool).  Computes the scaled residual
 * ||b - A x|| / ||b|| (||b|| replaced by 1 when it is at most eps(||b||)) of
 * a CSR system with every array (rowptr[n+1], colval, nzval, x[n], b[n]) and
 * the result (one double) in device memory.  Each row's sum follows its CSR
 * order and the two norms use the library's fixed reduction tree over the
 * rows in the order given, so for rows given in any order the result equals
 * the residual xcal_solve_system reports up to rounding; it is the same value
 * bit for bit only when the rows come in the library's storage order.  Runs on the
 * calling thread's current device, on `stream` (NULL = legacy stream),
 * without synchronising.  n is limited to 33,554,432 rows (larger n returns
 * XCAL_ERR_INVALID).  It allocates nothing: its scratch is a fixed ~256 KiB
 * device array inside the library, present on every GPU that loads it.  The
 * first call on a device resolves that array's address, so make it before
 * any stream capture.  Calls share the array: calls whose work overlaps on
 * the GPU race and must be serialised by the caller.  err/errlen (may be
 * NULL/0) receive a message on failure. */
int32_t xcal_residual_noalloc(int32_t n, const int32_t* rowptr, const int32_t* colval, const double* nzval,
                              const double* x, const double* b, double* result, void* stream, char* err,
                              int32_t errlen);

/* ---- bounded waits ----------------------------------------------------------
 * No counterpart in the reference.  The persistent kernels' grid barriers
 * poll a bounded number of times, then set an error flag and return, so a
 * block that never arrives becomes XCAL_ERR_TIMEOUT on the host, not a hung
 * GPU.  This check runs that path on purpose and without any fault: one
 * block waits at a barrier for a second block that is never launched, giving
 * up after spin_limit polls (1 .. 4,194,304; about 0.1 us each).  gave_up = 1
 * and flag_set = 1 when the wait ended by its limit; ran_after = 1 when a
 * kernel launched after it still ran (the context stayed usable). */
int32_t xcal_check_bounded_wait(xcal_ctx* ctx, int64_t spin_limit, int32_t* gave_up, int32_t* flag_set,
                                int32_t* ran_after);

/* ---- timers --------------------------------------------------------------*/
/* cumulative device time (ms) per phase since case creation:
 * [0] assembly+BCs, [1] U Krylov, [2] p Krylov, [3] gradients/interp/flux,
 * [4] residuals, [5] total iterate; returns the number of entries written */
int32_t xcal_get_timings(const xcal_case* cs, double* ms, int32_t n);
/* number of kernel launches issued by this library since it was loaded
 * (library-wide; cs may be NULL) */
int32_t xcal_get_launch_count(const xcal_case* cs, int64_t* count);
/* the cudaStream_t the case launches on (as void*), so a caller can record
 * its own CUDA events around library calls */
int32_t xcal_case_stream(const xcal_case* cs, void** stream);
/* per-kernel CUDA-event timing of the dominant kernels (off by default).
 * which: 0 = CG SpMV (+ p.Ap), 1 = BiCGSTAB SpMV, 2 = DILU sweep levels,
 *        3 = CG vector update (+ Jacobi apply and r.z when fused),
 *        4 = count only: every CG SpMV launch that did work (ms = 0),
 *        5 = persistent CG launches (ms; launches = CG iterations they ran).
 * ms = summed device time, launches = timed launches that did work.  Inside
 * the steady-state CUDA-graph chunks only sampled iterations are timed. */
int32_t xcal_case_set_profiling(xcal_case* cs, int32_t enable);
/* graph mode (off by default): each xcal_simple_iterate iteration /
 * xcal_piso_step step replays one CUDA graph captured on first use.  The
 * Krylov loops run as conditional WHILE nodes whose stopping tests are taken
 * on the device (at most itmax/4 + 2 loop bodies), so a step needs one host
 * synchronisation.  Results are identical to the default mode.  Per-kernel
 * profiling does not apply inside the graph. */
int32_t xcal_case_set_graph_mode(xcal_case* cs, int32_t enable);
/* persistent CG (on by default): a CG solve with Jacobi or no preconditioner
 * runs as one cooperative launch (grid barriers between the SpMV and update
 * phases, q kept on chip) whenever the system's tiles fit the GPU at once;
 * otherwise, and in graph mode, the two-kernel loop runs.  Same results.
 * mode: 0 off; 1 on: a system of at most 16 tiles of 2048 rows runs as one
 * thread-block cluster (hardware cluster barriers), a larger one in the
 * widest cooperative block form whose blocks are co-resident (1024, 512 or
 * 256 threads); 2 = the cluster form only, 256 / 512 / 1024 = that
 * cooperative form only, 4 / 5 = one block of 1024 / 512 threads per SM,
 * each owning every 148th tile (its q in shared memory: up to 12 FP64 / 25
 * FP32 tiles per block) (each falls back to the two-kernel loop when it
 * does not fit). */
int32_t xcal_case_set_persistent(xcal_case* cs, int32_t mode);
/* Krylov report of the last solve of each system (Ux, Uy, Uz, p, k, omega,
 * wall distance): iterations (mixed precision: inner iterations over all
 * defect-correction steps) and status -- 0 running, 1 solved, 2 stopped at
 * itmax, 3 zero curvature, 4 breakdown, 5 zero right-hand side -- and the
 * number of solves since the case was created that stopped at itmax.
 * solve_system! warns "Maximum number of iterations reached!" for those
 * (src/Solve/Solve_1_api.jl:302); the library keeps going as the reference
 * does and reports them here.  Any pointer may be NULL. */
int32_t xcal_case_solve_report(const xcal_case* cs, int32_t* iters7, int32_t* status7, int64_t* itmax_hits);
/* Mixed precision, CG with the Jacobi preconditioner: form of the FP32 inner
 * solves.  No counterpart in the reference (its Krylov.jl solves have no
 * inner precision).  0 (default) = CG on the Jacobi-scaled system
 * M^1/2 A M^1/2 (the same iteration in exact arithmetic, deterministic, its
 * own reduction order) where the system fits one block per SM, else as 1;
 * 1 = the FP32 form of the FP64 path's kernels; 2 + v = the scaled-system
 * kernel with v = s + 4 g + 8 w: s (0..3) its launch shape (768 or 1024
 * threads per block, with or without the next row's slot loads issued
 * early), g = 1 the iterate and the direction kept in global memory instead
 * of shared memory, w = 1 per-slice slot widths even where one uniform width
 * would do.  Shapes with the same thread count, g and w change where data
 * lives, not the results (768-thread shapes agree bit for bit, as do
 * 1024-thread ones).  All meet the same stopping tests; results agree within
 * the mixed-precision tolerance. */
int32_t xcal_case_set_inner_cg(xcal_case* cs, int32_t mode);
/* launch-shape autotuner (runs on first use, or now): out6 = for U then p,
 * (SpMV rows per thread [0 = canonical tile kernel], SpMV block size, DILU
 * form [0 one launch per level, 1 one-block sweeps, 2 one cooperative launch
 * over every level]).  The choices never change a result. */
int32_t xcal_case_tuning(xcal_case* cs, int32_t* out6);
/* DILU execution: 0 = autotuned (default), 1 = one-block sweeps,
 * 2 = one launch per level over level-ordered triangles, 3 = every level of
 * an application in one cooperative launch (a grid barrier between levels).
 * Same results, bit for bit. */
int32_t xcal_case_set_dilu_mode(xcal_case* cs, int32_t mode);
int32_t xcal_case_get_profile(const xcal_case* cs, int32_t which, double* ms, int64_t* launches);

/* ---- batching / serving --------------------------------------------------
 * A batch keeps many independent steady cases resident and advances them one
 * SIMPLE iteration per call in lockstep.  Each Krylov solve (U x, y, z, then
 * p) is one batched solve over all cases: a single launch per Krylov kernel
 * covers every case's tiles (block-diagonal system, per-case offsets), with
 * per-case Krylov scalars -- a case's results are the same alone, in any
 * batch, and through xcal_simple_iterate.  Cases must share the precision
 * mode, solvers and preconditioners.  Cases enter and leave between
 * iterations; admission is bounded by max_cases and a device-memory budget.
 * (The reference has no counterpart: it solves one case per process.) */
/* device bytes a case will hold (mesh + fields + matrices + workspaces),
 * from its sizes, before it is created; an upper bound */
int32_t xcal_footprint_estimate(int64_t n_cells, int64_t n_faces, int64_t n_bfaces, int32_t precision,
                                int32_t dilu_U, int32_t dilu_p, int64_t* bytes);
/* device bytes held by a created case and by its mesh */
int32_t xcal_case_footprint(const xcal_case* cs, int64_t* case_bytes, int64_t* mesh_bytes);
int32_t xcal_batch_create(xcal_ctx* ctx, int32_t max_cases, int64_t budget_bytes, xcal_batch** out);
int32_t xcal_batch_destroy(xcal_batch* b);
/* admit a case (it then runs on the batch's stream); charge_bytes <= 0
 * charges its measured footprint.  XCAL_ERR_BUSY when full or over budget.
 * An admitted case's mixed-precision inner CG takes the canonical form
 * (xcal_case_set_inner_cg mode 1), the batch's own, for good. */
int32_t xcal_batch_add(xcal_batch* b, xcal_case* cs, int64_t charge_bytes);
int32_t xcal_batch_remove(xcal_batch* b, xcal_case* cs);
int32_t xcal_batch_info(const xcal_batch* b, int32_t* n_cases, int64_t* used_bytes, int64_t* budget_bytes);
/* host wall time (ms) spent by xcal_batch_simple_iterate so far:
 * [face loops + corrections, U solves, p solve, total] */
int32_t xcal_batch_timings(const xcal_batch* b, double* ms4);
/* position of a case in the batch's order (the row of its results) */
int32_t xcal_batch_case_index(const xcal_batch* b, const xcal_case* cs, int32_t* index);
/* one SIMPLE iteration of every admitted case; res [n_cases*4] receives the
 * scaled residuals (Ux, Uy, Uz, p) and converged [n_cases] the per-case
 * convergence test of Solvers_1_SIMPLE.jl:222-240: 1 converged, 0 not yet,
 * or XCAL_ERR_DIVERGED for a case whose residual was NaN/Inf.  Such a case
 * has left the batch when the call returns (its budget charge is released;
 * the caller destroys or inspects it); the other cases are unaffected and
 * the call returns XCAL_OK.  Rows follow the order before the call (either
 * array may be NULL). */
int32_t xcal_batch_simple_iterate(xcal_batch* b, double* res, int32_t* converged);

#ifdef __cplusplus
}
#endif
#endif /* XCAL_B200_H */
