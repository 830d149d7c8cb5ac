"""
    XCALibre_B200Ext

Package extension of XCALibre.jl that runs the incompressible SIMPLE/PISO hot
path on an NVIDIA B200 (sm_100a) through `libxcal_b200`, a C ABI
(`include/xcal_b200.h`).  It is the sibling of `XCALibre_CUDAExt`
(`ext/XCALibre_CUDAExt.jl:18-156` of XCALibre.jl): XCALibre loads it when
the trigger package `XCALibreB200` is loaded, which defines the backend type
`B200Backend(; device=0, precision=:fp64, graph=false)` and the path of the
shared library (`XCALibreB200.libxcal`).  In XCALibre's `Project.toml`:

    [weakdeps]
    XCALibreB200 = "<uuid of the package shipping libxcal_b200.so>"
    [extensions]
    XCALibre_B200Ext = "XCALibreB200"

With `Hardware(backend=B200Backend(), workgroup=32)` in the configuration,
`run!(model, config; pref, ncorrectors, inner_loops)` keeps its signature and
its user API (`Physics`, `assign`, `SolverSetup`, `Schemes`, `Runtime`,
`Configuration`, `initialise!`): `simple!` / `piso!` below marshal the mesh,
boundary conditions and configuration once, run every iteration in the
library, and copy U, p (and k, omega, kl, nut where the model has them) back
into the model's fields.  Residual histories come back as the reference returns
them, `(Ux=..., Uy=..., Uz=..., p=...)`.

The structs below mirror the C structs field for field; `__init__` compares
their `sizeof` and `fieldoffset`s with the library's own
(`xcal_abi_layout`), so a mirror that drifts from the header fails at load
time instead of passing wrong memory.  Host arrays are caller-owned and read
only during each call (`GC.@preserve`); device memory belongs to the library
handles.
"""
module XCALibre_B200Ext

if isdefined(Base, :get_extension)
    using XCALibreB200
else
    using ..XCALibreB200
end

using XCALibre
using XCALibreB200: B200Backend, libxcal

# ---------------------------------------------------------------------------
# constants of include/xcal_b200.h
# ---------------------------------------------------------------------------
const XCAL_OK = Int32(0)
const XCAL_ERR_NOT_CONVERGED = Int32(-4)

const BC_DIRICHLET = Int32(1)
const BC_DIRICHLET_FUNCTION = Int32(2)
const BC_WALL = Int32(3)
const BC_ZEROGRADIENT = Int32(4)
const BC_EXTRAPOLATED = Int32(5)
const BC_EMPTY = Int32(6)
const BC_SYMMETRY = Int32(7)
const BC_NEUMANN = Int32(8)
const BC_PERIODIC = Int32(9)
const BC_PERIODIC_PARENT = Int32(10)
const BC_OMEGA_WALL = Int32(11)
const BC_K_WALL = Int32(12)
const BC_NUT_WALL = Int32(13)

const TIME_STEADY, TIME_EULER = Int32(0), Int32(1)
const DIV_LINEAR, DIV_UPWIND, DIV_LUST = Int32(0), Int32(1), Int32(2)
const GRAD_GAUSS, GRAD_MIDPOINT = Int32(0), Int32(1)
const LIMITER_NONE, LIMITER_CELL, LIMITER_FACE, LIMITER_MFACE = Int32(0), Int32(1), Int32(2), Int32(3)
const SOLVER_CG, SOLVER_BICGSTAB = Int32(0), Int32(1)
const PRECOND_NONE, PRECOND_JACOBI, PRECOND_DILU = Int32(0), Int32(1), Int32(2)
const TURB_LAMINAR, TURB_SMAGORINSKY, TURB_KOMEGA, TURB_KOMEGA_SST, TURB_KEQUATION, TURB_KOMEGA_LKE =
    Int32(0), Int32(1), Int32(2), Int32(3), Int32(4), Int32(5)
const PREC_FP64, PREC_MIXED = Int32(0), Int32(1)
const ALGO_SIMPLE, ALGO_PISO = Int32(0), Int32(1)

const FIELD_U, FIELD_P, FIELD_NUT, FIELD_K, FIELD_OMEGA, FIELD_KL =
    Int32(0), Int32(1), Int32(9), Int32(15), Int32(16), Int32(21)

# xcal_abi_layout selectors
const LAYOUT_MESH_DESC, LAYOUT_BC, LAYOUT_SOLVER_SETUP, LAYOUT_SCHEMES, LAYOUT_CONFIG =
    Int32(0), Int32(1), Int32(2), Int32(3), Int32(4)

# ---------------------------------------------------------------------------
# C structs, field for field
# ---------------------------------------------------------------------------
# xcal_mesh_desc: the Mesh3 contract (Mesh_0_types.jl:28-205), SoA, 0-based
struct MeshDesc
    n_cells::Int32
    n_faces::Int32
    n_bfaces::Int32
    face_owner::Ptr{Int32}
    face_neigh::Ptr{Int32}
    face_centre::Ptr{Float64}
    face_normal::Ptr{Float64}
    face_e::Ptr{Float64}
    face_area::Ptr{Float64}
    face_delta::Ptr{Float64}
    face_weight::Ptr{Float64}
    cell_centre::Ptr{Float64}
    cell_volume::Ptr{Float64}
    cell_faces_offset::Ptr{Int32}
    cell_faces::Ptr{Int32}
    cell_nsign::Ptr{Int32}
    cell_neighbours::Ptr{Int32}
    boundary_cellsID::Ptr{Int32}
    n_patches::Int32
    patch_start::Ptr{Int32}
    patch_count::Ptr{Int32}
    dim::Int32
end

# xcal_bc: one boundary condition of one field on one patch
struct BCDesc
    type::Int32
    patch::Int32
    value::NTuple{3,Float64}
    face_values::Ptr{Float64}
    face_map::Ptr{Int32}
    distance::NTuple{3,Float64}
    partner_patch::Int32
    wall::NTuple{5,Float64}
end

# xcal_solver_setup: SolverSetup (Solve_1_api.jl:8-83)
struct SolverSetupDesc
    solver::Int32
    precond::Int32
    convergence::Float64
    relax::Float64
    atol::Float64
    rtol::Float64
    itmax::Int32
    smoother_loops::Int32
    smoother_omega::Float64
end

# xcal_schemes: Schemes (Solve_1_api.jl:205-211)
struct SchemesDesc
    time::Int32
    divergence::Int32
    gradient::Int32
    limiter::Int32
    limiter_level::Float64
end

# xcal_config: Configuration + Physics as the hot path reads them
struct ConfigDesc
    algorithm::Int32
    turbulence::Int32
    nu::Float64
    smagorinsky_C::Float64
    les_delta_distance::Float64
    les_delta_power::Float64
    U_schemes::SchemesDesc
    p_schemes::SchemesDesc
    U_solver::SolverSetupDesc
    p_solver::SolverSetupDesc
    iterations::Int32
    dt::Float64
    has_pref::Int32
    pref::Float64
    inner_loops::Int32
    ncorrectors::Int32
    precision::Int32
    inner_rtol::Float64
    n_bc_U::Int32
    n_bc_p::Int32
    n_bc_nut::Int32
    bc_U::Ptr{BCDesc}
    bc_p::Ptr{BCDesc}
    bc_nut::Ptr{BCDesc}
    kw_beta_star::Float64
    kw_alpha1::Float64
    kw_beta1::Float64
    kw_sigma_k::Float64
    kw_sigma_omega::Float64
    k_schemes::SchemesDesc
    omega_schemes::SchemesDesc
    k_solver::SolverSetupDesc
    omega_solver::SolverSetupDesc
    n_bc_k::Int32
    n_bc_omega::Int32
    bc_k::Ptr{BCDesc}
    bc_omega::Ptr{BCDesc}
    sst_beta2::Float64
    sst_sigma_k2::Float64
    sst_sigma_omega2::Float64
    y_schemes::SchemesDesc
    y_solver::SolverSetupDesc
    n_bc_y::Int32
    bc_y::Ptr{BCDesc}
    keq_ck::Float64
    keq_ce::Float64
    lke_Tu::Float64
    kl_schemes::SchemesDesc
    kl_solver::SolverSetupDesc
    n_bc_kl::Int32
    bc_kl::Ptr{BCDesc}
end

# xcal_term / xcal_source: one operator / source of an equation built with
# the DSL (ModelFramework_0_types.jl:18-100), for xcal_equation_create
struct TermDesc
    op::Int32
    scheme::Int32
    sign::Float64
    flux::Ptr{Float64}
    value::Float64
end

struct SourceDesc
    sign::Float64
    field::Ptr{Float64}
    value::Float64
end

const LAYOUT_TERM, LAYOUT_SOURCE = Int32(7), Int32(8)

const MIRRORS = ((LAYOUT_MESH_DESC, MeshDesc), (LAYOUT_BC, BCDesc), (LAYOUT_SOLVER_SETUP, SolverSetupDesc),
                 (LAYOUT_SCHEMES, SchemesDesc), (LAYOUT_CONFIG, ConfigDesc), (LAYOUT_TERM, TermDesc),
                 (LAYOUT_SOURCE, SourceDesc))

# the library's sizeof and field offsets against the mirrors
function check_layouts()
    buf = zeros(Int64, 64)
    for (which, T) in MIRRORS
        n = ccall((:xcal_abi_layout, libxcal), Int32, (Int32, Ptr{Int64}, Int32), which, buf, length(buf))
        n == fieldcount(T) + 1 || error("libxcal_b200: $(T) has $(fieldcount(T)) fields, the library $(n - 1)")
        buf[1] == sizeof(T) || error("libxcal_b200: sizeof($(T)) = $(sizeof(T)), the library's is $(buf[1])")
        for k in 1:fieldcount(T)
            buf[k + 1] == fieldoffset(T, k) ||
                error("libxcal_b200: $(T).$(fieldname(T, k)) at $(fieldoffset(T, k)), the library's at $(buf[k + 1])")
        end
    end
end

__init__() = check_layouts()

# ---------------------------------------------------------------------------
# handles and errors
# ---------------------------------------------------------------------------
last_error(ctx::Ptr{Cvoid}) = unsafe_string(ccall((:xcal_last_error, libxcal), Cstring, (Ptr{Cvoid},), ctx))

function check(ctx::Ptr{Cvoid}, code::Integer)
    code == XCAL_OK && return nothing
    error("libxcal_b200 error $(code): $(ctx == C_NULL ? "" : last_error(ctx))")
end

# ---------------------------------------------------------------------------
# mesh: AoS Face3D / Cell, 1-based -> SoA, 0-based
# ---------------------------------------------------------------------------
function mesh_arrays(mesh)
    F = mesh.faces
    C = mesh.cells
    nb = length(mesh.boundary_cellsID)
    vec3(vs) = (a = Vector{Float64}(undef, 3 * length(vs));
                for (i, v) in enumerate(vs); a[3i - 2] = v[1]; a[3i - 1] = v[2]; a[3i] = v[3]; end; a)
    off = Vector{Int32}(undef, length(C) + 1)
    off[1] = 0
    for (i, c) in enumerate(C)
        off[i + 1] = off[i] + Int32(length(c.faces_range))
    end
    return (owner=Int32[f.ownerCells[1] - 1 for f in F],
            neigh=Int32[f.ownerCells[2] - 1 for f in F],
            face_centre=vec3([f.centre for f in F]),
            face_normal=vec3([f.normal for f in F]),
            face_e=vec3([f.e for f in F]),
            face_area=Float64[f.area for f in F],
            face_delta=Float64[f.delta for f in F],
            face_weight=Float64[f.weight for f in F],
            cell_centre=vec3([c.centre for c in C]),
            cell_volume=Float64[c.volume for c in C],
            cell_faces_offset=off,
            cell_faces=Int32.(mesh.cell_faces .- 1),
            cell_nsign=Int32.(mesh.cell_nsign),
            cell_neighbours=Int32.(mesh.cell_neighbours .- 1),
            boundary_cellsID=Int32.(mesh.boundary_cellsID .- 1),
            patch_start=Int32[first(b.IDs_range) - 1 for b in mesh.boundaries],
            patch_count=Int32[length(b.IDs_range) for b in mesh.boundaries],
            n_bfaces=nb,
            dim=mesh isa XCALibre.Mesh.Mesh2 ? Int32(2) : Int32(3))
end

# valid while `a` is preserved by the caller
function mesh_desc(mesh, a)
    MeshDesc(Int32(length(mesh.cells)), Int32(length(mesh.faces)), Int32(a.n_bfaces),
             pointer(a.owner), pointer(a.neigh), pointer(a.face_centre), pointer(a.face_normal),
             pointer(a.face_e), pointer(a.face_area), pointer(a.face_delta), pointer(a.face_weight),
             pointer(a.cell_centre), pointer(a.cell_volume), pointer(a.cell_faces_offset),
             pointer(a.cell_faces), pointer(a.cell_nsign), pointer(a.cell_neighbours),
             pointer(a.boundary_cellsID), Int32(length(a.patch_start)), pointer(a.patch_start),
             pointer(a.patch_count), a.dim)
end

# ---------------------------------------------------------------------------
# boundary conditions (after `assign`: bc.ID is the patch index, 1-based)
# ---------------------------------------------------------------------------
const BC_TYPES = Dict{Symbol,Int32}(
    :Dirichlet => BC_DIRICHLET, :DirichletFunction => BC_DIRICHLET_FUNCTION, :Wall => BC_WALL,
    :Zerogradient => BC_ZEROGRADIENT, :Extrapolated => BC_EXTRAPOLATED, :Empty => BC_EMPTY,
    :Symmetry => BC_SYMMETRY, :Neumann => BC_NEUMANN, :Periodic => BC_PERIODIC,
    :PeriodicParent => BC_PERIODIC_PARENT, :OmegaWallFunction => BC_OMEGA_WALL,
    :KWallFunction => BC_K_WALL, :NutWallFunction => BC_NUT_WALL)

bc_kind(bc) = get(BC_TYPES, nameof(typeof(bc))) do
    error("libxcal_b200: boundary condition $(nameof(typeof(bc))) is not on the B200 path")
end

value3(v::Number) = (Float64(v), 0.0, 0.0)
value3(v) = (Float64(v[1]), Float64(v[2]), length(v) > 2 ? Float64(v[3]) : 0.0)

# DirichletFunction: f(face.centre, time, index) per face of the patch,
# components interleaved (dirichletFunction.jl:39-118)
function face_values(bc, mesh, time, ncomp)
    r = mesh.boundaries[bc.ID].IDs_range
    out = Vector{Float64}(undef, ncomp * length(r))
    for (k, fID) in enumerate(r)
        v = bc.value(mesh.faces[fID].centre, time, fID)
        for c in 1:ncomp
            out[ncomp * (k - 1) + c] = ncomp == 1 ? Float64(v[1]) : Float64(v[c])
        end
    end
    out
end

# wall-function constants kappa, beta1, cmu^0.25, yPlusLam, E
wall5(v) = (Float64(v.kappa), Float64(v.beta1), Float64(v.cmu)^0.25, Float64(v.yPlusLam), Float64(v.E))

# the BCDesc table of one field, and the arrays it points into
function bc_table(bcs, mesh, time, ncomp)
    keep = Any[]
    out = BCDesc[]
    for bc in bcs
        t = bc_kind(bc)
        val = (0.0, 0.0, 0.0)
        fv = Ptr{Float64}(C_NULL)
        fmap = Ptr{Int32}(C_NULL)
        dist = (0.0, 0.0, 0.0)
        partner = Int32(-1)
        wall = (0.0, 0.0, 0.0, 0.0, 0.0)
        if t == BC_DIRICHLET_FUNCTION
            a = face_values(bc, mesh, time, ncomp)
            push!(keep, a)
            fv = pointer(a)
        elseif t == BC_PERIODIC || t == BC_PERIODIC_PARENT
            pv = bc.value
            m = Int32.(pv.face_map .- 1)
            push!(keep, m)
            fmap = pointer(m)
            dist = value3(pv.transform.distance)
            partner = Int32(pv.patchID - 1)
        elseif t == BC_OMEGA_WALL || t == BC_K_WALL || t == BC_NUT_WALL
            wall = wall5(bc.value)
        elseif t != BC_EMPTY && t != BC_ZEROGRADIENT && t != BC_SYMMETRY
            val = value3(bc.value)
        end
        push!(out, BCDesc(t, Int32(bc.ID - 1), val, fv, fmap, dist, partner, wall))
    end
    push!(keep, out)
    return out, keep
end

# ---------------------------------------------------------------------------
# solvers, schemes, physics
# ---------------------------------------------------------------------------
solver_kind(s) = s isa XCALibre.Solve.Cg ? SOLVER_CG :
                 s isa XCALibre.Solve.Bicgstab ? SOLVER_BICGSTAB :
                 error("libxcal_b200: solver $(typeof(s)) is not on the B200 path (Cg, Bicgstab)")

function precond_kind(p)
    p isa XCALibre.Solve.Jacobi && return PRECOND_JACOBI
    p isa XCALibre.Solve.DILU && return PRECOND_DILU
    error("libxcal_b200: preconditioner $(typeof(p)) is not on the B200 path (Jacobi, DILU)")
end

function solver_desc(s)
    loops, omega = Int32(0), 0.0
    if s.smoother !== nothing
        loops = Int32(s.smoother.loops)
        omega = Float64(s.smoother.omega)
    end
    SolverSetupDesc(solver_kind(s.solver), precond_kind(s.preconditioner), Float64(s.convergence),
                    Float64(s.relax), Float64(s.atol), Float64(s.rtol), Int32(s.itmax), loops, omega)
end
solver_desc(::Nothing) = SolverSetupDesc(SOLVER_CG, PRECOND_JACOBI, 1e-7, 1.0, 1e-15, 0.1, Int32(1000), Int32(0), 0.0)

time_kind(t) = t === XCALibre.Discretise.Euler ? TIME_EULER : TIME_STEADY
div_kind(d) = d === XCALibre.Discretise.Upwind ? DIV_UPWIND : d === XCALibre.Discretise.LUST ? DIV_LUST : DIV_LINEAR
grad_kind(g) = g === XCALibre.Discretise.Midpoint ? GRAD_MIDPOINT : GRAD_GAUSS

function schemes_desc(s)
    lim, level = LIMITER_NONE, 0.0
    if hasproperty(s, :limiter) && s.limiter !== nothing
        lname = nameof(typeof(s.limiter))
        if lname == :CellBased
            lim, level = LIMITER_CELL, Float64(s.limiter.level)
        elseif lname == :FaceBased
            lim = LIMITER_FACE
        elseif lname == :MFaceBased
            lim = LIMITER_MFACE
        else
            error("libxcal_b200: limiter $(typeof(s.limiter)) is not on the B200 path")
        end
    end
    SchemesDesc(time_kind(s.time), div_kind(s.divergence), grad_kind(s.gradient), lim, level)
end
schemes_desc(::Nothing) = SchemesDesc(TIME_STEADY, DIV_LINEAR, GRAD_GAUSS, LIMITER_NONE, 0.0)

getopt(nt, k) = hasproperty(nt, k) ? getproperty(nt, k) : nothing

"""
    config_desc(model, config; pref=nothing, inner_loops=0, ncorrectors=0, algorithm=ALGO_SIMPLE)

The `ConfigDesc` of a run, and the arrays its BC tables point into (keep them
alive, `GC.@preserve`, for the call that reads it).
"""
function config_desc(model, config; pref=nothing, inner_loops=0, ncorrectors=0, algorithm=ALGO_SIMPLE)
    (; solvers, schemes, runtime, hardware, boundaries) = config
    mesh = model.domain
    be = hardware.backend
    turb = model.turbulence
    tname = nameof(typeof(turb))
    tk = tname == :Laminar ? TURB_LAMINAR : tname == :Smagorinsky ? TURB_SMAGORINSKY :
         tname == :KOmega ? TURB_KOMEGA : tname == :KOmegaSST ? TURB_KOMEGA_SST :
         tname == :KEquation ? TURB_KEQUATION : tname == :KOmegaLKE ? TURB_KOMEGA_LKE :
         error("libxcal_b200: turbulence model $(tname) is not on the B200 path")
    time = 0.0
    keep = Any[]
    tab(f, nc) = (bcs = getopt(boundaries, f); bcs === nothing ? (BCDesc[], Any[]) : bc_table(bcs, mesh, time, nc))
    bU, kU = tab(:U, 3)
    bp, kp = tab(:p, 1)
    bnut, knut = tab(:nut, 1)
    bk, kk = tab(:k, 1)
    bw, kw = tab(:omega, 1)
    by, ky = tab(:y, 1)
    bkl, kkl = tab(:kl, 1)
    append!(keep, (bU, bp, bnut, bk, bw, by, bkl, kU, kp, knut, kk, kw, ky, kkl))
    ptr(v) = isempty(v) ? Ptr{BCDesc}(C_NULL) : pointer(v)
    C = tk == TURB_SMAGORINSKY ? Float64(turb.coeffs.C) : 0.0
    kwc = tk in (TURB_KOMEGA, TURB_KOMEGA_SST) ? turb.coeffs : nothing
    g(k) = kwc === nothing ? 0.0 : Float64(getproperty(kwc, k))
    gs(k) = (kwc === nothing || !hasproperty(kwc, k)) ? 0.0 : Float64(getproperty(kwc, k))
    sk1 = tk == TURB_KOMEGA_SST ? :σk1 : :σk
    sw1 = tk == TURB_KOMEGA_SST ? :σω1 : :σω
    desc = ConfigDesc(
        algorithm, tk, Float64(model.fluid.nu.values), C, 0.0, 0.0,
        schemes_desc(schemes.U), schemes_desc(schemes.p),
        solver_desc(solvers.U), solver_desc(solvers.p),
        Int32(runtime.iterations), Float64(Array(runtime.dt)[1]),
        Int32(pref === nothing ? 0 : 1), Float64(pref === nothing ? 0.0 : pref),
        Int32(inner_loops), Int32(ncorrectors),
        be.precision == :mixed ? PREC_MIXED : PREC_FP64, 0.0,
        Int32(length(bU)), Int32(length(bp)), Int32(length(bnut)), ptr(bU), ptr(bp), ptr(bnut),
        g(:β⁺), g(:α1), g(:β1), g(sk1), g(sw1),
        schemes_desc(getopt(schemes, :k)), schemes_desc(getopt(schemes, :omega)),
        solver_desc(getopt(solvers, :k)), solver_desc(getopt(solvers, :omega)),
        Int32(length(bk)), Int32(length(bw)), ptr(bk), ptr(bw),
        gs(:β2), gs(:σk2), gs(:σω2),
        schemes_desc(getopt(schemes, :y)), solver_desc(getopt(solvers, :y)),
        Int32(length(by)), ptr(by),
        tk == TURB_KEQUATION ? Float64(turb.coeffs.ck) : 0.0, tk == TURB_KEQUATION ? Float64(turb.coeffs.ce) : 0.0,
        tk == TURB_KOMEGA_LKE ? Float64(turb.Tu) : 0.0,
        schemes_desc(getopt(schemes, :kl)), solver_desc(getopt(solvers, :kl)), Int32(length(bkl)), ptr(bkl))
    return desc, keep
end

# ---------------------------------------------------------------------------
# run!: simple! and piso! on Hardware{<:B200Backend}
# ---------------------------------------------------------------------------
const B200Config = XCALibre.Simulate.Configuration{SC,SL,RT,<:XCALibre.Simulate.Hardware{<:B200Backend}} where {SC,SL,RT}

function set_field!(ctx, case, id, values)
    check(ctx, ccall((:xcal_case_set_field, libxcal), Int32, (Ptr{Cvoid}, Int32, Ptr{Float64}, Int64),
                     case, id, values, length(values)))
end
function get_field!(ctx, case, id, out)
    check(ctx, ccall((:xcal_case_get_field, libxcal), Int32, (Ptr{Cvoid}, Int32, Ptr{Float64}, Int64),
                     case, id, out, length(out)))
    out
end

function b200_run(model, config, algorithm; pref=nothing, ncorrectors=0, inner_loops=0)
    be = config.hardware.backend
    mesh = model.domain
    ctx = Ref{Ptr{Cvoid}}(C_NULL)
    check(C_NULL, ccall((:xcal_ctx_create, libxcal), Int32, (Int32, Ref{Ptr{Cvoid}}), Int32(be.device), ctx))
    dmesh = Ref{Ptr{Cvoid}}(C_NULL)
    case = Ref{Ptr{Cvoid}}(C_NULL)
    try
        arrays = mesh_arrays(mesh)
        GC.@preserve arrays begin
            md = Ref(mesh_desc(mesh, arrays))
            check(ctx[], ccall((:xcal_mesh_upload, libxcal), Int32, (Ptr{Cvoid}, Ref{MeshDesc}, Ref{Ptr{Cvoid}}),
                               ctx[], md, dmesh))
        end
        desc, keep = config_desc(model, config; pref=pref, inner_loops=inner_loops, ncorrectors=ncorrectors,
                                 algorithm=algorithm)
        GC.@preserve keep begin
            cd = Ref(desc)
            check(ctx[], ccall((:xcal_case_create, libxcal), Int32,
                               (Ptr{Cvoid}, Ptr{Cvoid}, Ref{ConfigDesc}, Ref{Ptr{Cvoid}}), ctx[], dmesh[], cd, case))
        end
        (; U, p) = model.momentum
        set_field!(ctx[], case[], FIELD_U, vcat(U.x.values, U.y.values, U.z.values))
        set_field!(ctx[], case[], FIELD_P, Vector{Float64}(p.values))
        # the turbulence fields the model has (k, omega, kl, nut)
        tfields = [(s, id) for (s, id) in ((:k, FIELD_K), (:omega, FIELD_OMEGA), (:kl, FIELD_KL), (:nut, FIELD_NUT))
                   if hasproperty(model.turbulence, s)]
        for (s, id) in tfields
            set_field!(ctx[], case[], id, Vector{Float64}(getproperty(model.turbulence, s).values))
        end
        be.graph && check(ctx[], ccall((:xcal_case_set_graph_mode, libxcal), Int32, (Ptr{Cvoid}, Int32), case[], 1))
        n = Int32(config.runtime.iterations)
        res = zeros(Float64, 4 * n)
        done = Ref{Int32}(0)
        if algorithm == ALGO_SIMPLE
            conv = Ref{Int32}(0)
            check(ctx[], ccall((:xcal_simple_iterate, libxcal), Int32,
                               (Ptr{Cvoid}, Int32, Ptr{Float64}, Ref{Int32}, Ref{Int32}), case[], n, res, done, conv))
            conv[] == 1 && @info "Simulation converged in $(done[]) iterations!"
        else
            courant = zeros(Float64, n)
            check(ctx[], ccall((:xcal_piso_step, libxcal), Int32,
                               (Ptr{Cvoid}, Int32, Ptr{Float64}, Ptr{Float64}, Ref{Int32}), case[], n, res, courant,
                               done))
        end
        nC = length(mesh.cells)
        Uh = get_field!(ctx[], case[], FIELD_U, Vector{Float64}(undef, 3 * nC))
        U.x.values .= @view Uh[1:nC]
        U.y.values .= @view Uh[nC+1:2nC]
        U.z.values .= @view Uh[2nC+1:3nC]
        p.values .= get_field!(ctx[], case[], FIELD_P, Vector{Float64}(undef, nC))
        for (s, id) in tfields
            getproperty(model.turbulence, s).values .= get_field!(ctx[], case[], id, Vector{Float64}(undef, nC))
        end
        # solve_system! warns for every solve that stopped at itmax
        # (Solve_1_api.jl:302); the library counts them
        hits = Ref{Int64}(0)
        check(ctx[], ccall((:xcal_case_solve_report, libxcal), Int32, (Ptr{Cvoid}, Ptr{Int32}, Ptr{Int32}, Ref{Int64}),
                           case[], C_NULL, C_NULL, hits))
        hits[] > 0 && @warn "Maximum number of iterations reached! ($(hits[]) Krylov solves stopped at itmax)"
        R = reshape(res, 4, :)[:, 1:done[]]
        return (Ux=R[1, :], Uy=R[2, :], Uz=R[3, :], p=R[4, :])
    finally
        case[] == C_NULL || ccall((:xcal_case_destroy, libxcal), Int32, (Ptr{Cvoid},), case[])
        dmesh[] == C_NULL || ccall((:xcal_mesh_destroy, libxcal), Int32, (Ptr{Cvoid},), dmesh[])
        ccall((:xcal_ctx_destroy, libxcal), Int32, (Ptr{Cvoid},), ctx[])
    end
end

# Solvers_1_SIMPLE.jl:28-43 / Solvers_2_PISO.jl:25-38, for the B200 backend
function XCALibre.Solvers.simple!(model, config::B200Config; output=XCALibre.VTK(), pref=nothing, ncorrectors=0,
                                  inner_loops=0)
    b200_run(model, config, ALGO_SIMPLE; pref=pref, ncorrectors=ncorrectors, inner_loops=inner_loops)
end

function XCALibre.Solvers.piso!(model, config::B200Config; output=XCALibre.VTK(), pref=nothing, ncorrectors=0,
                                inner_loops=2)
    b200_run(model, config, ALGO_PISO; pref=pref, ncorrectors=ncorrectors, inner_loops=inner_loops)
end

end # module
