// case.hpp -- host objects behind the C ABI handles.
#pragma once
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>

#include "kernels.hpp"
#include "xcal_internal.hpp"

// A context may be used from several host threads at once (serving sets up
// cases on worker threads while another thread iterates), so each thread
// keeps its own last error message: a failure on one thread never shows up
// as another thread's error.  Elements of an unordered_map keep their address
// across insertions, so the pointer xcal_last_error returns stays valid until
// the same thread's next failing call on this context.
struct xcal_ctx {
    int device = 0;
    void set_error(const std::string& msg) {
        std::lock_guard<std::mutex> g(mu);
        errors[std::this_thread::get_id()] = msg;
    }
    const char* last_error() {
        std::lock_guard<std::mutex> g(mu);
        auto it = errors.find(std::this_thread::get_id());
        return it == errors.end() ? "" : it->second.c_str();
    }

   private:
    std::mutex mu;
    std::unordered_map<std::thread::id, std::string> errors;
};

namespace xcal {

// Mesh3 in HBM plus host copies needed to derive per-equation structures
struct DevMesh {
    int nC = 0, nF = 0, nB = 0, nI = 0;
    int dim = 3;  // 2 for a Mesh2
    // storage order: perm[s] = original index stored at s, inv = its inverse
    // (cells); fperm/finv likewise for faces (boundary faces are not moved)
    std::vector<int> perm, inv, fperm, finv;
    // host copies (0-based)
    std::vector<int> owner, neigh, cf_off, cf_face, cf_nb, bcell, bf_off, bf_face, bcells, patch_start, patch_count;
    std::vector<signed char> cf_sign;
    std::vector<double> vol, area, delta, ccx, ccy, ccz, fcx, fcy, fcz, nxh, nyh, nzh, ex, ey, ez;
    // device
    DBuf<int> d_owner, d_neigh, d_cf_off, d_cf_face, d_cf_nb, d_bf_off, d_bf_face, d_bcell, d_bcells;
    DBuf<signed char> d_cf_sign;
    DBuf<double> d_area, d_delta, d_weight, d_Sx, d_Sy, d_Sz, d_nx, d_ny, d_nz, d_Ef, d_vol;
    DBuf<int> d_perm, d_inv, d_fperm, d_finv;  // storage <-> original order (field transfer)
    size_t bytes = 0;  // device bytes held
    MeshView view() const;
};

// Level-ordered SELL-32 copy of one triangle's off-diagonal entries (DILU
// sweeps of large systems): position k of the level order (the row
// rows[k]) holds that row's strictly lower (or upper) entries in the row's
// own order, so the rows of one level read their slots coalesced.  `src` maps
// each slot to the matrix slot whose value it mirrors; values (and, for the
// lower triangle, dinv = 1/D of each slot's column) are refreshed before
// each DILU-preconditioned solve.
struct LevelSell {
    long nslots = 0;
    DBuf<int> slice, col, src;
    DBuf<int> tsrc;   // lower triangle: slot of the transposed entry a_ji (DILU factor)
    DBuf<int> dslot;  // lower triangle: diagonal slot of each position's row (DILU factor)
    DBuf<unsigned char> cnt;
    DBuf<double> val, dinv;
    DBuf<float> val32, dinv32;
};

struct Equation;
// device view of one level-ordered triangle of E (tri 0 lower, 1 upper) in
// value type T (refreshed by Case::dilu_refresh)
template <class T>
LevelView<T> level_view(const Equation& E, int tri);
// the level-ordered lower triangle as the DILU factor reads it
LevelDView level_d_view(const Equation& E);

struct Equation {
    int n = 0;
    long nnz = 0;
    long nnz_csr = 0;                       // entries without SELL padding
    std::vector<int> slice, colval, diag;   // host pattern (SELL-32, storage rows)
    std::vector<unsigned char> len;
    DBuf<int> d_slice, d_colval, d_diag, d_trans, d_cf_slot, d_fslot;
    DBuf<unsigned char> d_len;
    int base(int r) const { return slice[r / SELL_C] + r % SELL_C; }
    DBuf<double> nz, nz0, diag0, P;
    DBuf<float> nz32, P32;  // mixed precision: FP32 copies for the inner solves
    // mixed precision, CG + Jacobi: off-diagonal slots of the Jacobi-scaled
    // system (built at first use; values refreshed per solve)
    DBuf<int> f_slice, f_col, f_map;
    DBuf<unsigned char> f_len;
    DBuf<float> f_val;
    bool fold_built = false;
    bool fold_uniform_ok = true;  // the layout rule the storage was built with
    int f_W = 0;  // uniform slice width of the folded storage (0: per-slice widths)
    FoldView fold_view() const { return FoldView{n, f_slice.p, f_len.p, f_col.p, f_val.p, f_W}; }
    FoldMut fold_mut() { return FoldMut{n, f_slice.p, f_len.p, f_col.p, f_map.p, f_val.p}; }
    DBuf<double> b[3];
    // DILU level schedules (rows grouped by dependency level)
    DBuf<int> d_lower_rows, d_upper_rows;
    std::vector<int> lower_off, upper_off;
    std::vector<int> h_lower_rows, h_upper_rows;  // host copies (batched level lists)
    DBuf<int> d_lower_off, d_upper_off;           // level offsets (one-block sweeps)
    LevelSell lsell, usell;                       // level-ordered triangles (level-kernel sweeps)
    // launch choices (autotune.cu); neither changes any result
    bool use_block = false;   // DILU as one-block sweeps (default: n <= DILU_BLOCK_MAX_ROWS)
    bool use_grid = false;    // else as one cooperative launch over every level (k_dilu_grid)
    SpmvShape spmv_shape;     // BiCGSTAB SpMV row mapping / block size
    bool dilu_block() const { return use_block; }
    bool has_periodic = false;
    CSRView view() const;
    int find(int i, int j) const;  // slot or -1
};

// the CSR pattern, slot maps and (need_dilu) DILU level structures of an
// equation on mesh m (periodic BCs add their partner entries); the BC table
// of a field (E: the equation whose periodic slots it resolves, or null)
void build_equation(Equation& E, const DevMesh& m, const std::vector<xcal_bc>& bcs, int nvec, bool need_dilu,
                    cudaStream_t s);
struct BCTable;
void build_bc_table(BCTable& T, const DevMesh& m, const xcal_bc* bcs, int nbc, int ncomp, const Equation* E,
                    cudaStream_t s);

struct BCTable {
    std::vector<xcal_bc> src;  // as given (pointers not retained)
    std::vector<signed char> type;
    std::vector<double> val;
    DBuf<signed char> d_type;
    DBuf<double> d_val, d_pw, d_pwn, d_pEf, d_pDelta, d_pwdelta;
    DBuf<int> d_peer_face, d_peer_cell, d_pNN, d_pNP, d_pPN, d_pe_off, d_pe_face;
    std::vector<int> h_pNP, h_pPN;  // periodic off-diagonal slots (parent faces; -1 elsewhere)
    bool has_periodic = false;
    BCView view() const;
};

struct KrylovWS {
    DBuf<double> x, dx, r, z, p, q, v, s, t, part0, part1;
    DBuf<float> fx, fr, fz, fp, fq, fv, fs, ft, fd;  // mixed precision inner vectors
    DBuf<double> fpart;  // folded inner CG: block partials (2 x FOLD_MAX_BLOCKS)
    DBuf<float2> frp;    // folded inner CG: two buffers of n (r, p_old) pairs
    DBuf<unsigned int> bar;  // persistent CG: grid-barrier state (count, generation)
    DBuf<int> err;           // persistent CG: a barrier wait gave up
    DBuf<KScalars> S;  // [2]: U, p
};

// work vectors of one Krylov solve
template <class T>
struct KrylovVecs {
    T *x, *r, *z, *p, *q, *v, *s, *t;
};

struct Case {
    xcal_ctx* ctx = nullptr;
    const DevMesh* mesh = nullptr;
    xcal_config cfg{};
    size_t bytes = 0;  // device bytes held (excluding the mesh)
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    BCTable bcU, bcP, bcNut, bcK, bcOmega, bcY, bcKl;
    Equation U, P;
    KrylovWS ws;
    // fields
    DBuf<double> nonorth;  // non-orthogonal correctors: per internal face w, e, T (7 x nI)
    DBuf<double> midR;     // Midpoint gradients: per internal face rf - 0.5 (rP + rN) (3 x nI)
    DBuf<double> limD;     // CellBased limiter: fc - cc per cell_faces entry (3 x 2 nI)
    DBuf<int> limOrd;      // MFaceBased: each cell's cell_faces entries in ascending reference face id
    DBuf<double> Uc[3], p, mdot, nueff, gradp[3], gradU[9], rD, Hv[3], divHv, nut, nutf, Uf[3], pf, rDf, Delta, prev,
        courant, dx13, resbuf, cmax, io;  // io: staging of one field component in the original order
    // RANS{KOmega}: k, omega, production / dissipation per cell, a scratch
    // copy for bound!, and the omega wall cells (storage ids) with, per cell,
    // y = delta of its constraining face, kappa, beta1, cmu^0.25, yPlusLam
    DBuf<double> kfld, omega, Pk, Pw, Dk, Dw, kwtmp, wpar;
    // RANS{KOmegaSST}: wall distance (and its potential), F1, F2, Omega, the
    // second omega Si coefficient, grad k, grad omega, a face scratch
    DBuf<double> yw, yphi, F1b, F2b, Omb, D2b, gkv[3], gwv[3], fscr;
    // RANS{KOmegaLKE}: kl, its source and Si coefficient, the per-cell flow
    // quantities of one turbulence! call (div U, S2, |U|, Re_lambda; Omega in
    // Omb, the cross diffusion in D2b), the intermittency gamma, the cell
    // diffusivity of the equation being set up and its face interpolation
    DBuf<double> kl, PkL, DkL, S2b, normUb, divUb, ReLb, gam, nueffS, fmu;
    double lke_eta = 0.0;  // 0.02974 tanh(59.79 Tu^1.191 + 1.65e-13)
    DBuf<int> wcell;
    int nwall = 0;
    // KWallFunction cells (last face in BC / face order) and NutWallFunction
    // faces, with kappa, cmu^0.25, yPlusLam, E per entry
    DBuf<int> kwcell, kwface, nwface;
    DBuf<double> kwpar, nwpar;
    int nkwall = 0, nnutwall = 0;
    double res_k = 0.0, res_omega = 0.0, res_kl = 0.0;
    bool initialised = false;
    int iteration = 0;
    double time = 0.0;
    int last_iters[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // Ux, Uy, Uz, p, k, omega, wall distance, kl
    // Krylov status (KS_*) of each system's last solve, and how many solves
    // since creation stopped at itmax (Solve_1_api.jl:302 warns on those)
    int last_status[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long itmax_hits = 0;
    void note_status(int gk, int status) {
        last_status[gk] = status;
        if (status == KS_TIRED) ++itmax_hits;
    }
    // timing
    double ms[6] = {0, 0, 0, 0, 0, 0};
    long long launches = 0;
    cudaEvent_t ev[8];
    KScalars* h_S = nullptr;  // pinned host mirror (2 entries)
    double* h_res = nullptr;  // pinned
    // optional per-kernel event timing (xcal_case_set_profiling)
    bool profiling = false;
    std::vector<cudaEvent_t> pev;  // pairs, reused per polling chunk
    double prof_ms[6] = {0, 0, 0, 0, 0, 0};
    long long prof_n[6] = {0, 0, 0, 0, 0, 0};
    int persistent_cg = 1;  // CG (Jacobi / none) as one cooperative launch: 0 off, 1 auto width, else the width
    // mixed-precision inner CG with Jacobi: 0 = on the Jacobi-scaled system
    // (cg_folded.cu) where it fits, 1 = the canonical FP32 kernels, 2 + v =
    // the scaled-system kernel with v = form (bits 0-1, launch shape) + 4 (x
    // and p kept in global memory) + 8 (per-slice slot widths even where the
    // uniform width would do); every v gives the same results as v & 3
    int inner_cg = 0;
    // inner_cg = 2 + s + 4 g + 8 w: form s, x/p in global memory (g),
    // per-slice slot widths (w)
    int fold_form() const { return inner_cg >= 2 ? (inner_cg - 2) & 3 : FOLD_DEFAULT_FORM; }
    bool fold_smem() const { return inner_cg < 2 || !((inner_cg - 2) & 4); }
    bool fold_uniform_ok() const { return inner_cg < 2 || !((inner_cg - 2) & 8); }
    void set_inner_cg(int mode);  // drops a captured step graph of the other form
    int dilu_mode = 0;          // 0 = autotuned / size rule, 1 = one-block sweeps, 2 = per-level kernels,
                                // 3 = one cooperative launch over every level
    // whether a cooperative kernel may be launched on the case stream now
    // (not capturing, or capturing where the driver runs such nodes)
    bool coop_ok_here();
    void prof_reserve(int pairs);
    // Steady-state polling chunks of a Krylov solve (32 CG / 8 BiCGSTAB
    // iterations) replay as CUDA graphs: every pointer they use is fixed for
    // the life of the case, so each graph is captured once per equation
    // component (BiCGSTAB reads the component's right-hand side).  The
    // profiled variant carries event-record nodes around sampled iterations
    // (those with c % 8 == 4).
    struct ChunkGraph {
        cudaGraphExec_t exec = nullptr;
        long long launches = 0;  // kernels per replay
    };
    ChunkGraph chunk_graph[7][2];  // [Ux, Uy, Uz, p, k, omega, wall distance][plain, profiled]
    cudaEvent_t gev[7][12] = {};   // event nodes of the profiled graphs
    template <class F>
    void replay_chunk(ChunkGraph& g, F&& body);

    Case(xcal_ctx* c, const DevMesh* m, const xcal_config* cfg);
    ~Case();

    // steps (each mirrors a reference function)
    void initial_calculations();
    void discretise(int eqn);
    void apply_bcs(int eqn, int comp);
    void relax_U(int comp);
    void bc_relax_U(int comp);
    void set_reference();
    void update_precond(int eqn);
    double solve_system(int eqn, int comp, int* iters);
    void solve_equation_U(double res[3]);
    double solve_equation_p();
    void pressure_predictor(bool with_H);
    void H();
    void flux_divergence();
    void build_nonorth(const DevMesh& m, cudaStream_t s);
    void build_midpoint(const DevMesh& m, cudaStream_t s);
    void build_limiter(const DevMesh& m, cudaStream_t s);
    void smooth(int eqn, int comp);
    // one linear solve: its system, setup, field, right-hand side, graph-mode
    // result slot, device-scalars slot and per-system index (k and omega use
    // the p system's storage, as the reference's equations share it, and
    // k's preconditioner type, RANS_kOmega.jl:77-85)
    struct SolveRef {
        Equation* E;
        xcal_solver_setup SS;
        double* field;
        const double* b;
        int slot, kslot, gk;
    };
    SolveRef solve_ref(int eqn, int comp);
    double solve_system_ref(const SolveRef& R, int* iters, bool fp64);
    void update_precond_E(Equation& E, int precond);
    void build_wall_table(const DevMesh& m);
    void komega();
    void kequation();  // turbulence!(::KEquationModel) after grad U (LES_KEquation.jl:134-186)
    void komega_lke();  // turbulence!(::KOmegaLKEModel) after grad U (RANS_kOmegaLKE.jl:262-474)
    bool sst() const { return cfg.turbulence == XCAL_TURB_KOMEGA_SST; }
    bool lke() const { return cfg.turbulence == XCAL_TURB_KOMEGA_LKE; }
    bool has_y() const { return sst() || lke(); }  // a wall distance field
    bool rans_kw() const { return cfg.turbulence == XCAL_TURB_KOMEGA || sst() || lke(); }
    bool keq() const { return cfg.turbulence == XCAL_TURB_KEQUATION; }
    bool has_k() const { return rans_kw() || keq(); }  // a k field and equation
    void scalar_grad(const double* phi, const BCTable& T, int scheme, double* const g[3]);
    void wall_distance();
    void nonorth_correct();
    void nonorth_correctors(double& rp);
    void explicit_relaxation_p(double a);
    void grad_p();
    void correct();
    void turbulence();
    double max_courant();
    bool simple_iteration(double res[4]);
    double piso_step(double res[4]);

    // helpers
    MeshView mv() const { return mesh->view(); }
    double* field_comp(int field, int comp, long& count);
    void sync();
    template <class T>
    void dilu_ldiv(Equation& E, const T* nz, const T* D, const T* b, T* out, const KScalars* S);
    template <class T>
    void apply_M(Equation& E, int ptype, const T* nz, const T* P, const T* in, T* out, const KScalars* S);
    void dilu_refresh(Equation& E, bool fp32);
    template <class T>
    void krylov_iterate(Equation& E, const xcal_solver_setup& SS, const T* nz, const T* P, const T* c, const T* r0,
                        const KrylovVecs<T>& V, KScalars* S, KScalars* hS, int gk);
    void solve_mixed(Equation& E, const xcal_solver_setup& SS, double* field, const double* b, KScalars* S,
                     KScalars* hS, int gk, int* iters);
    // mixed precision, CG + Jacobi: whether the inner solves of E run on the
    // Jacobi-scaled system (cg_folded.cu), and one such inner solve of the
    // scaled defect in V.r (host-polled; field corrected by the kernel)
    bool use_fold(const Equation& E, const xcal_solver_setup& SS, bool captured) const;
    void fold_iterate(Equation& E, double* field, const KrylovVecs<float>& V, KScalars* S, KScalars* hS, int gk);
    int last_outer[7] = {0, 0, 0, 0, 0, 0, 0};  // mixed: defect-correction steps of the last solve per system
    bool tuned = false;
    void autotune();  // launch-shape autotuner (autotune.cu), once per case

    // ---- graph mode: one SIMPLE iteration / PISO step captured as a CUDA
    // graph; the Krylov (and defect-correction) loops are conditional WHILE
    // nodes driven by device-side stopping tests, so a step needs no host
    // round trip until its residuals are read.
    enum { GRES_U = 0, GRES_P = 3, GRES_CO = 4, GRES_K = 5, GRES_OMEGA = 6, GRES_KL = 7, GRES_N = 8 };
    DBuf<double> gres;          // per-step results: U x,y,z and p residuals, max Courant
    DBuf<int> giters;           // (iterations, status) of the step's 4 solves
    DBuf<unsigned int> cmax_ctr;
    DBuf<unsigned long long> dlaunch;  // kernels run inside WHILE bodies (graph mode)
    long long step_top_kernels = 0;    // kernels of a step graph outside WHILE bodies
    bool graph_mode = false;    // xcal_case_set_graph_mode
    bool capturing = false;     // the step functions are being captured
    cudaStream_t side[2] = {nullptr, nullptr};  // capture streams of WHILE bodies
    int side_depth = 0;
    cudaGraphExec_t step_graph = nullptr;
    long long step_graph_launches = 0;
    int* h_iters = nullptr;     // pinned mirror of giters
    unsigned long long* h_launch = nullptr;
    int* h_perr = nullptr;      // pinned: persistent CG error flag after a graph replay
    long long body_kernels_captured = 0;
    long long last_body_kernels = 0;  // kernels captured into the last WHILE body
    void simple_body(double r3[3], double& rp, bool timed);
    void piso_body(double r3[3], double& rp);
    void set_graph_mode(bool on);
    void courant_to_slot();
    template <class F>
    void capture_while(F&& body);
    void solve_captured(int eqn, int comp);
    template <class T>
    void krylov_start(Equation& E, const xcal_solver_setup& SS, const T* nz, const T* P, const T* c, const T* r0,
                      const KrylovVecs<T>& V, KScalars* S);
    template <class T>
    void krylov_step(Equation& E, const xcal_solver_setup& SS, const T* nz, const T* P, const T* c,
                     const KrylovVecs<T>& V, KScalars* S, cudaEvent_t* ev6, bool in_capture);
    void capture_step();
    void run_step_graph(double res[4], double* courant);
};

}  // namespace xcal

struct xcal_mesh {
    xcal_ctx* ctx = nullptr;
    std::unique_ptr<xcal::DevMesh> m;
};

struct xcal_case {
    std::unique_ptr<xcal::Case> c;
};
