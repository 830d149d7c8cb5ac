// kernels.hpp -- host-side launchers of the device kernels.
#pragma once
#include "xcal_internal.hpp"

namespace xcal {

// flags of launch_bc_relax_U: start from the assembled diagonal, apply the
// boundary conditions, apply the implicit relaxation
enum { BCR_DIAG0 = 1, BCR_BC = 2, BCR_RELAX = 4 };

// finite-volume kernels (kernels_fv.cu)
void launch_assemble_U(cudaStream_t s, const MeshView& m, const CSRView& A, const double* mdot, const double* nueff,
                       const double* const U[3], const double* const g[3], double* nz, double* diag0,
                       double* const b[3], int time_scheme, int div_scheme, double dt);
void launch_assemble_p(cudaStream_t s, const MeshView& m, const CSRView& A, const double* rDf, const double* divHv,
                       double* nz, double* b);
void launch_bc_relax_U(cudaStream_t s, const MeshView& m, const CSRView& A, const BCView& bc, int comp,
                       int div_scheme, double* nz, const double* diag0, double* b, const double* mdot,
                       const double* nueff, const double* const U[3], double alpha, int flags);
void launch_bc_p(cudaStream_t s, const MeshView& m, const CSRView& A, const BCView& bc, double* nz, double* b,
                 const double* rDf, const double* p);
void launch_set_reference(cudaStream_t s, const CSRView& A, double* nz, double* b, double pref, int row);
void launch_interp_U(cudaStream_t s, const MeshView& m, const BCView& bc, const double* const U[3],
                     double* const Uf[3], double* mdot);
void launch_interp_scalar(cudaStream_t s, const MeshView& m, const BCView& bc, const double* phi, double* phif,
                          double* nueff, double nu);
void launch_interp_rD(cudaStream_t s, const MeshView& m, const BCView& bcU, const double* rD, double* rDf);
void launch_fill(cudaStream_t s, double* a, double v, long n);
void launch_green_gauss(cudaStream_t s, const MeshView& m, const double* phif, double* const g[3]);
void launch_green_gauss_tensor(cudaStream_t s, const MeshView& m, double* const Uf[3], double* const g[9],
                               const double* Delta, double* nut);
void launch_div(cudaStream_t s, const MeshView& m, const double* psif, double* out);
// Midpoint gradient face passes (internal faces; R: Case::build_midpoint)
void launch_mid_scalar(cudaStream_t s, const MeshView& m, const double* phi, double* phif);
void launch_mid_vector(cudaStream_t s, const MeshView& m, const double* const U[3], double* const Uf[3]);
void launch_mid_correct_scalar(cudaStream_t s, const MeshView& m, const double* R, const double* phi,
                               const double* const g[3], double* phif);
void launch_mid_correct_vector(cudaStream_t s, const MeshView& m, const double* R, const double* const U[3],
                               const double* const g[9], double* const Uf[3]);
// CellBased gradient limiter of grad F, F a scalar field or one component of
// U with its row of grad U (D: Case::build_limiter)
// limit_gradient!(FaceBased) of a scalar's gradient (3 arrays) / a vector's
// (9 arrays, one limiter per cell for all nine); D as for launch_limit_cell
void launch_limit_face_scalar(cudaStream_t s, const MeshView& m, const double* D, const double* F,
                              double* const g[3]);
void launch_limit_face_vector(cudaStream_t s, const MeshView& m, const double* D, const double* const U[3],
                              double* const g[9]);
void launch_limit_cell(cudaStream_t s, const MeshView& m, const double* D, const double* F, double* const g[3],
                       double level);
// MFaceBased: a cell's internal faces in ascending face order (ord: the
// cell_faces entries so sorted), each correcting the gradient in turn
void launch_limit_mface_scalar(cudaStream_t s, const MeshView& m, const int* ord, const double* D, const double* F,
                               double* const g[3]);
void launch_limit_mface_vector(cudaStream_t s, const MeshView& m, const int* ord, const double* D,
                               const double* const U[3], double* const g[9]);
// RANS{KOmega}: sources, k / omega assembly, BCs + relaxation, the omega
// wall rows, bound!, nut = k / omega; nueff = nu + nutf
void launch_kw_sources(cudaStream_t s, int nC, const double* const g[9], const double* nut, const double* omega,
                       double* Pk, double* Pw, double* Dk, double* Dw, double alpha1, double beta1, double beta_star);
// (F1 null: constant sigma; F1 set: sigma blended with sigma2 (k-omega SST);
// D2 / si2: a second Si term with sign d2_sign: omega's cross diffusion in
// k-omega SST (+) and k-omega LKE (-), KEquation's 2/3 div U (+))
void launch_assemble_scalar(cudaStream_t s, const MeshView& m, const CSRView& A, const double* mdot,
                            const double* nutf, double nu, double sigma, const double* F1, double sigma2,
                            const double* phi, const double* D, const double* D2, const double* P, double* nz,
                            double* b, int time_scheme, int div_scheme, double dt, double d2_sign = 1.0);
void launch_bc_relax_scalar(cudaStream_t s, const MeshView& m, const CSRView& A, const BCView& bc, double* nz,
                            double* b, const double* mdot, const double* nutf, double nu, double sigma,
                            const double* F1, double sigma2, int si2, const double* phi, double alpha,
                            int div_scheme);
// k-omega SST: cell fields, nut, and the wall distance from phi and grad phi
void launch_sst_fields(cudaStream_t s, int nC, const double* const g[9], const double* const gk[3],
                       const double* const gw[3], const double* k, const double* omega, const double* nut,
                       const double* yw, double* F1, double* F2, double* Om, double* Pk, double* Pw, double* Dk,
                       double* Dw, double* D2, double bs, double al1, double b1, double b2, double sw2, double nu);
void launch_sst_nut(cudaStream_t s, int nC, const double* k, const double* omega, const double* F2, const double* Om,
                    double al1, double* nut);
void launch_walldist(cudaStream_t s, int nC, const double* phi, const double* const g[3], double* y);
// wall functions: KWallFunction production per wall cell, NutWallFunction
// nutf (and nueff) per wall face; par: kappa, cmu^0.25, yPlusLam, E
void launch_kwall_production(cudaStream_t s, int nw, const MeshView& m, const int* cell, const int* face,
                             const double* par, const double* k, const double* const U[3], double nu, double* Pk);
void launch_nutwall(cudaStream_t s, int nw, const MeshView& m, const int* face, const double* par, const double* k,
                    double nu, double* nutf, double* nueff);
void launch_omega_constrain(cudaStream_t s, int nw, const CSRView& A, const int* wcell, const double* par,
                            const double* k, double nu, double* nz, double* b);
void launch_bound(cudaStream_t s, const MeshView& m, const double* old, double* v);
void launch_kw_nut(cudaStream_t s, int nC, const double* k, const double* omega, double* nut);
// LES{KEquation}: the k equation's cell sources (Pk, Si coefficients) and nut
void launch_keq_sources(cudaStream_t s, int nC, const double* const g[9], const double* nut, const double* k,
                        const double* Delta, double ce, double* Pk, double* Dk, double* Dw);
void launch_keq_nut(cudaStream_t s, int nC, const double* k, const double* Delta, double ck, double* nut);
// RANS{KOmegaLKE} (RANS_kOmegaLKE.jl:270-460): the cell loops of one
// turbulence! call over these buffers (n_cells each)
struct LkeView {
    const double* g[9];   // grad U, row-major (d u_a / d x_b at 3a + b)
    const double* U[3];
    const double* gk[3];  // grad k, grad omega (cross diffusion)
    const double* gw[3];
    const double* y;      // wall distance
    const double* kl;
    const double* k;
    const double* omega;
    double *divU, *S2, *Om, *normU, *ReL, *gam;  // per-cell flow quantities
    double *Pk, *Pw, *PkL, *Dk, *Dw, *DkL, *D2;   // sources and Si coefficients
    double* nueffS;  // the equation being set up: its cell diffusivity
    double* nut;
    int nC;
    double nu, eta;
};
void launch_lke_fields(cudaStream_t s, const LkeView& V);  // flow quantities, gamma, the kl equation
void launch_lke_omega(cudaStream_t s, const LkeView& V);   // the omega equation
void launch_lke_k(cudaStream_t s, const LkeView& V);       // fv and the k equation
void launch_lke_nut(cudaStream_t s, const LkeView& V);     // nut = nuts + nuL
void launch_nueff(cudaStream_t s, int nF, const double* nutf, double* nueff, double nu);
// Smagorinsky nut = Delta |S| from a stored grad U
void launch_smag_nut(cudaStream_t s, int nC, const double* const g[9], const double* Delta, double* nut);
// non-orthogonal correction of the pressure right-hand side (t: Case::build_nonorth)
void launch_nonorth_correct(cudaStream_t s, const MeshView& m, const double* t, const double* p,
                            const double* const g[3], const double* rDf, double* b);
void launch_rD_remove_H(cudaStream_t s, const MeshView& m, const CSRView& A, const double* nz,
                        const double* const U[3], const double* const g[3], double* const b[3], double* rD,
                        double* const H[3], int do_H);
void launch_H(cudaStream_t s, const MeshView& m, const CSRView& A, const double* nz, const double* const U[3],
              const double* const b[3], double* const H[3]);
void launch_correct_mdot(cudaStream_t s, const MeshView& m, const CSRView& A, const BCView& bcp, const double* nz,
                         const double* p, const double* rDf, double* mdot);
void launch_correct_U(cudaStream_t s, int n, double* const H[3], const double* const g[3], const double* rD,
                      double* const U[3]);
void launch_relax_explicit(cudaStream_t s, int n, double* phi, const double* phi0, double alpha);
void launch_gather(cudaStream_t s, long n, const double* src, const int* idx, double* dst);
void launch_courant_max(cudaStream_t s, int n, const double* const U[3], const double* dx, double dt, double* part,
                        unsigned int* counter, double* out);

// Krylov kernels (kernels_krylov.cu).  Templates are instantiated for
// T = double (plain FP64 path) and T = float (mixed-precision inner solves).
void kr_init_resid(cudaStream_t s, const CSRView& A, const double* nz, const double* b, const double* field,
                   double* dx, double* x, double* r);
// mixed precision: d = (float)(b - A*field), x = 0; field += x; dst = (float)src
void kr_defect(cudaStream_t s, const CSRView& A, const double* nz, const double* b, const double* field, float* d,
               float* x);
void kr_correct(cudaStream_t s, int n, double* field, const float* x);
void kr_to_float(cudaStream_t s, long n, const double* src, float* dst);
template <class T>
void kr_spmv(cudaStream_t s, const CSRView& A, const T* nz, const T* x, T* y, const KScalars* S);
// launch shape of an SpMV without a reduction: rows_per_thread 0 = the
// canonical tile kernel (kr_spmv), else 1/2/4 rows per thread, `block` threads
struct SpmvShape {
    int rows_per_thread = 0;
    int block = 256;
};
template <class T>
void kr_spmv_shaped(cudaStream_t s, const SpmvShape& sh, const CSRView& A, const T* nz, const T* x, T* y,
                    const KScalars* S);
template <class T>
void kr_jacobi_apply(cudaStream_t s, int n, const T* P, const T* r, T* z, const KScalars* S);
template <class T>
void kr_copy(cudaStream_t s, int n, const T* a, T* b, const KScalars* S);
template <class T>
void kr_cg_start(cudaStream_t s, int n, const T* r, const T* z, T* p, KScalars* S, double* part);
// CG direction p_k lives in P0 (k even) / P1 (k odd); p_0 = z is stored in P0
template <class T>
void kr_cg_spmv(cudaStream_t s, const CSRView& A, const T* nz, const T* z, T* P0, T* P1, T* q, KScalars* S,
                double* part);
template <class T>
void kr_cg_update(cudaStream_t s, int n, T* x, const T* P0, const T* P1, T* r, const T* q, T* z, const T* P,
                  int jacobi_fused, KScalars* S, double* part);
template <class T>
void kr_cg_rz(cudaStream_t s, int n, const T* r, const T* z, KScalars* S, double* part);
// The whole CG loop in one cooperative launch (Jacobi: jacobi = 1, P = inverse
// diagonal; no preconditioner: jacobi = 0, z aliases r).  Returns false,
// launching nothing, when the system's tiles cannot all be co-resident.
// bar: 2 words of barrier state, err: set when a barrier wait gave up.
template <class T>
bool kr_cg_persist(cudaStream_t s, const CSRView& A, const T* nz, const T* P, int jacobi, T* x, T* r, T* z, T* P0,
                   T* P1, KScalars* S, double* part, double* part2, unsigned int* bar, int* err, int max_iters,
                   int width = 0, int pf_kb = 0, bool reset_err = true);
// width: 0 = the cluster form where the system has at most
// PERSIST_CLUSTER_MAX tiles, else the widest cooperative form that fits;
// PERSIST_CLUSTER_ONLY = the cluster form only; 256 / 512 / 1024 = that
// cooperative form only.  false: nothing launched (does not fit).
constexpr int PERSIST_CLUSTER_ONLY = 2;
constexpr int PERSIST_COOP_ONLY = 3;  // the widest cooperative form that fits, never the cluster form
// one block per SM, each owning every G-th tile (1024 or 512 threads; the
// block's q in shared memory: at most PERSIST_MT_SMEM bytes)
constexpr int PERSIST_MT1024 = 4;
constexpr int PERSIST_MT512 = 5;
constexpr int PERSIST_MT_SMEM = 200 * 1024;
// whether this device and driver run a cooperative kernel captured into a
// CUDA graph (in_while: inside the body of a conditional WHILE node); found
// out once per process by capturing and running a one-block no-op that way
bool kr_coop_capture_ok(bool in_while);
// the same for a kernel launched as thread-block clusters
bool kr_cluster_capture_ok(bool in_while);
// Persistent CG widths: 1024 / 512 threads per block (wide form, systems of
// at most 1 / 2 tiles per SM) or RED_THREADS (narrow form).  The launchers
// take the widest form whose co-resident capacity covers the tiles.
constexpr int PERSIST_WIDTHS[3] = {1024, 512, 256};
struct PersistCaps {
    bool init = false;
    int cap[3] = {0, 0, 0};  // co-resident blocks per width on this device
};
// index into PERSIST_WIDTHS of the form to launch for ntiles tiles, or -1
// (kernels: the three instantiations in PERSIST_WIDTHS order; width 0 = the
// widest that fits, else only that width)
int persist_pick(PersistCaps& c, const void* const kernels[3], int ntiles, int width = 0);
// cooperative launch of kernel (width index w) over ntiles blocks; false
// (capacity lowered, nothing launched) when the device refuses the size
bool persist_launch(PersistCaps& c, int w, const void* kernel, int ntiles, cudaStream_t s, void** args);
// Cluster form of the persistent CG (1024-thread blocks): a system of at
// most PERSIST_CLUSTER_MAX tiles runs as one thread-block cluster.  The
// cluster size for `tiles`: the smallest power of two >= tiles that the
// device schedules for this kernel, or 0 (too many tiles / not schedulable).
constexpr int PERSIST_CLUSTER_MAX = 16;
int persist_cluster_size(const void* kernel, int tiles);
// launch nclusters clusters of C blocks (one system each)
void persist_cluster_launch(const void* kernel, int C, int nclusters, cudaStream_t s, void** args);
void kr_finish(cudaStream_t s, int n, const double* x, const double* dx, double* field);
template <class T>
void kr_bicg_start(cudaStream_t s, int n, const T* c, const T* r, T* p, KScalars* S, double* part0, double* part1);
template <class T>
void kr_bicg_alpha(cudaStream_t s, int n, const T* c, const T* v, KScalars* S, double* part);
template <class T>
void kr_bicg_s(cudaStream_t s, int n, const T* r, const T* v, const T* p, T* sv, T* x, const KScalars* S);
template <class T>
void kr_bicg_omega(cudaStream_t s, int n, const T* t, const T* sv, KScalars* S, double* part0, double* part1);
template <class T>
void kr_bicg_xr(cudaStream_t s, int n, T* x, const T* sv, const T* t, T* r, const T* c, KScalars* S, double* part0,
                double* part1);
template <class T>
void kr_bicg_p(cudaStream_t s, int n, const T* r, const T* v, T* p, const KScalars* S);
void kr_jacobi_update(cudaStream_t s, const CSRView& A, const double* nz, double* P);
// apply_smoother!(JacobiSmoother) (Smoothers_jacobi.jl:88-110): `loops`
// sweeps x -> xt, each copied back into x
void kr_jacobi_smooth(cudaStream_t s, const CSRView& A, const double* nz, const double* b, double* x, double* xt,
                      int loops, double omega);
void kr_dilu_D(cudaStream_t s, const int* rows, int nrows, const CSRView& A, const double* nz, double* D);
template <class T>
void kr_dilu_fwd(cudaStream_t s, const int* rows, int nrows, const CSRView& A, const T* nz, const T* D, const T* b,
                 T* y, const KScalars* S);
template <class T>
void kr_dilu_bwd(cudaStream_t s, const int* rows, int nrows, const CSRView& A, const T* nz, const T* D, T* x,
                 const KScalars* S);
// DILU level sweeps over level-ordered triangles (positions k0..k1 of one
// level); the forward sweep reads dinv (T(1)/D of each slot's column,
// kr_level_dinv) instead of dividing per entry -- the same values
template <class T>
void kr_dilu_fwd_lv(cudaStream_t s, int k0, int k1, const int* rows, const int* slice, const unsigned char* cnt,
                    const int* col, const T* val, const T* dinv, const T* b, T* y, const KScalars* S);
// dinv[e] = T(1) / D[col[e]] for every slot of a level-ordered triangle
template <class T>
void kr_level_dinv(cudaStream_t s, long nslots, const int* col, const T* D, T* dinv);
template <class T>
void kr_dilu_bwd_lv(cudaStream_t s, int k0, int k1, const int* rows, const int* slice, const unsigned char* cnt,
                    const int* col, const T* val, const T* D, T* x, const KScalars* S);
template <class T>
void kr_gather_vals(cudaStream_t s, long n, const int* src, const T* vals, T* dst);
// small systems (n <= DILU_BLOCK_MAX_ROWS): whole sweeps in one block
// the lower triangle in level order, as the DILU factor reads it: per
// position k its row, the diagonal slot of that row (dslot), and per entry
// (in the row's own order) the column, the slot of a_ij (src) and of a_ji
// (tsrc) in the matrix
struct LevelDView {
    const int* rows;
    const int* off;
    int nlev;
    const int* slice;
    const unsigned char* cnt;
    const int* col;
    const int* src;
    const int* tsrc;
    const int* dslot;
};
// the D factor over the level-ordered lower triangle: one block (D staged in
// shared memory when it fits), or one cooperative launch over the grid with
// a grid barrier between levels (false: nothing launched); each row's
// arithmetic that of kr_dilu_D
void kr_dilu_D_lv_block(cudaStream_t s, int n, const LevelDView& L, const double* nz, double* D);
bool kr_dilu_D_lv_grid(cudaStream_t s, const LevelDView& L, const double* nz, double* D, unsigned int* bar,
                       int* err);
void kr_dilu_D_block(cudaStream_t s, const int* rows, const int* off, int nlev, const CSRView& A, const double* nz,
                     double* D);
// one triangle in level order, as the one-block sweep reads it: level l is
// positions off[l] .. off[l+1] of rows[]; position k keeps cnt[k] slots at
// slice[k/32] + k%32 + 32 j (values val, and for the lower triangle dinv)
template <class T>
struct LevelView {
    const int* rows;
    const int* off;
    int nlev;
    const int* slice;
    const unsigned char* cnt;
    const int* col;
    const T* val;
    const T* dinv;
};
// y in shared memory for systems of at most this many bytes of y
constexpr int DILU_SMEM_MAX_BYTES = 200 * 1024;
template <class T>
void kr_dilu_block(cudaStream_t s, int n, const LevelView<T>& lo, const LevelView<T>& up, const T* D, const T* b,
                   T* y, const KScalars* S);
// a whole DILU application (every level of both sweeps) as one cooperative
// launch with a grid barrier between levels; false (nothing launched) when
// the device cannot run it.  bar: 2 words zeroed here; err: set when a
// barrier wait gave up (the result is then incomplete)
template <class T>
bool kr_dilu_grid(cudaStream_t s, const LevelView<T>& lo, const LevelView<T>& up, const T* D, const T* b, T* y,
                  unsigned int* bar, int* err, const KScalars* S);
// the DILU factor D (every level of the lower triangle) as one cooperative
// launch; rows/off: the lower triangle's level lists on the device
bool kr_dilu_D_grid(cudaStream_t s, const int* rows, const int* off, int nlev, const CSRView& A, const double* nz,
                    double* D, unsigned int* bar, int* err);
void kr_residual(cudaStream_t s, const CSRView& A, const double* nz, const double* x, const double* b, KScalars* S,
                 double* part0, double* part1, double* out);
// device-driven solve control of graph mode (conditional WHILE nodes)
void kr_ks_init(cudaStream_t s, KScalars* S, double atol, double rtol, int itmax, int mixed, double inner_rtol);
// body_kernels: kernels of one loop body (excluding WHILE bodies nested in
// it), added to *launches each time the body runs
void kr_loop_cond(cudaStream_t s, cudaGraphConditionalHandle h, KScalars* S, int cap, int body_kernels,
                  unsigned long long* launches);
void kr_set_cond(cudaStream_t s, cudaGraphConditionalHandle h, unsigned int v);
void kr_outer_prep(cudaStream_t s, KScalars* S);
void kr_correct_masked(cudaStream_t s, int n, double* field, const float* x, const KScalars* S);
void kr_outer_cond(cudaStream_t s, cudaGraphConditionalHandle h, KScalars* S, int max_outer, int body_kernels,
                   unsigned long long* launches);
void kr_record(cudaStream_t s, const KScalars* S, int* out);

// ---- mixed precision: FP32 inner CG on the Jacobi-scaled system (cg_folded.cu)
// Off-diagonal entries of Ahat = M^1/2 A M^1/2 (M = diag(1/|a_ii|)) in
// SELL-32 slices over the storage rows: entry m of row i at slice[i/32] +
// i%32 + 32 m; len[i] = the row's off-diagonal count, bit 7 set when its
// diagonal is negative (ahat_ii = -1); map = the slot of the same entry in
// the equation's own SELL storage.  W > 0: every slice has the same width
// W (slice[s] = 32 W s) and a row's slots past its count hold its own column
// and a zero value, so a kernel may read all W without the row's count.
struct FoldView {
    int n;
    const int* slice;
    const unsigned char* len;
    const int* col;
    const float* val;
    int W;
};
struct FoldMut {
    int n;
    const int* slice;
    unsigned char* len;
    const int* col;
    const int* map;
    float* val;
};
// kernel forms of the folded CG (block size / software pipelining over rows;
// cg_folded.cu)
constexpr int FOLD_NFORMS = 4;
// most blocks of a folded-CG launch (one per SM); its two partial buffers
// hold this many doubles each
constexpr int FOLD_MAX_BLOCKS = 1024;
constexpr int FOLD_DEFAULT_FORM = 2;  // 768 threads, next row's loads early (fastest at 2.1M rows, no spills)
struct FoldShape {
    int form = 0, nt = 0, blocks = 0, rows = 0, smem = 0;
    bool smem_p = false, smem_x = false;
};
// blocks = 0: the system is too large for the folded CG.  vectors_in_smem:
// keep x and p in shared memory where they fit (else both in global memory;
// the same arithmetic either way)
FoldShape fold_shape(int n, int form = FOLD_DEFAULT_FORM, bool vectors_in_smem = true);
// rp[].x = (float)(sqrt(P) (b - A field)) in FP64 (P: FP64 Jacobi inverse
// diagonal); rp[].y is left as it is
void kr_fold_defect(cudaStream_t s, const CSRView& A, const double* nz, const double* b, const double* field,
                    const double* P, float2* rp);
// gamma = <r, r> over rp[].x and cg!'s start tests into S (part: one double
// per reduction tile)
void kr_fold_start(cudaStream_t s, int n, const float2* rp, KScalars* S, double* part);
// scaled off-diagonal values and diagonal signs from the FP64 matrix and P
void kr_fold_scale(cudaStream_t s, const FoldMut& F, const double* nz, const int* diag, const double* P);
// the whole inner solve after kr_fold_defect(RP0) and kr_fold_start, with field +=
// sqrt(P) xhat applied at its end unless S->outer_conv; false: too large
// (nothing launched).  xg: an n-float buffer used when x does not fit
// shared memory; part, part2: FOLD_MAX_BLOCKS doubles each.  RP0, RP1: n
// (r, p_old) pairs each, swapped every iteration.
bool kr_cgf_persist(cudaStream_t s, const FoldView& F, float2* RP0, float2* RP1, float* xg, double* field,
                    const double* Pj, KScalars* S, double* part, double* part2, unsigned int* bar, int* err,
                    int max_iters, bool reset_err = true, int form = FOLD_DEFAULT_FORM,
                    bool vectors_in_smem = true);

}  // namespace xcal
