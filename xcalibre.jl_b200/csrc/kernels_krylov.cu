// kernels_krylov.cu -- Krylov solves of the hot path.
//
// CG and BiCGSTAB follow Krylov.jl 0.10 (cg!, bicgstab!; called from
// src/Solve/Solve_1_api.jl:286-289 with warm start, M = preconditioner,
// ldiv = true for DILU).  All scalars live on the device; each reduction is a
// canonical tile tree finished by the last block of the kernel, which also
// takes the algorithm's scalar decisions (step sizes, stopping tests), so the
// host only polls a `done` flag between chunks of iterations.
//
// Every Krylov kernel is a template over the value type T of the matrix and
// the work vectors.  T = double is the plain FP64 path (its arithmetic is the
// oracle's, operation for operation).  T = float is the inner solver of the
// mixed-precision mode: FP32 matrix values, vectors and row sums, with dot
// products accumulated in FP64 and the step scalars kept in FP64 on the
// device and rounded to FP32 where they scale a vector.
#include <algorithm>
#include <map>
#include <mutex>

#include "kernels.hpp"
#include "krylov_bodies.cuh"

namespace xcal {

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// kernels (grid = one canonical tile per block, RED_THREADS threads)
// ---------------------------------------------------------------------------
// r = b - A*x0, x = 0, dx = x0 (warm start: Krylov.jl kaxpby!(n,1,b,-1,r))
__global__ void __launch_bounds__(RED_THREADS, 8) k_init_resid(CSRView A, const double* __restrict__ nz,
                                                            const double* __restrict__ b,
                                                            const double* __restrict__ field, double* dx, double* x,
                                                            double* r) {
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < A.n) {
            r[i] = b[i] - row_dot(A, nz, field, i);
            x[i] = 0.0;
            dx[i] = field[i];
        }
    }
}

// Defect of a mixed-precision correction step: d = b - A*x in FP64, stored
// rounded to FP32 as the inner right-hand side; the inner iterate starts at 0.
__global__ void __launch_bounds__(RED_THREADS, 8) k_defect(CSRView A, const double* __restrict__ nz,
                                                        const double* __restrict__ b,
                                                        const double* __restrict__ field, float* d, float* x) {
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < A.n) {
            d[i] = (float)(b[i] - row_dot(A, nz, field, i));
            x[i] = 0.0f;
        }
    }
}

// field += correction (FP64 accumulation of the FP32 inner solution)
__global__ void k_correct(int n, double* field, const float* __restrict__ x) {
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) field[i] = field[i] + (double)x[i];
    }
}

// dst = (float) src, any length
__global__ void k_to_float(long n, const double* __restrict__ src, float* dst) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        dst[i] = (float)ld_stream(src + i);
}

// y = A*x (plain SpMV, early exit when the solve is done)
template <class T>
__global__ void __launch_bounds__(RED_THREADS, 8) k_spmv(CSRView A, const T* __restrict__ nz,
                                                      const T* __restrict__ x, T* y, const KScalars* S) {
    spmv_body<T>(grid_tiles(), A, nz, x, y, S);
}

// y = A*x with a free row mapping (no reduction rides on this SpMV): thread g
// of the grid computes rows g, g + G, ..., R of them (G = threads in the
// grid).  The row sums are row_dot's, so every shape gives the same y; the
// shape (R, block size) is chosen by the autotuner.
template <class T, int R>
__global__ void k_spmv_rows(CSRView A, const T* __restrict__ nz, const T* __restrict__ x, T* y, const KScalars* S) {
    if (S && S->done) return;
    const int G = gridDim.x * blockDim.x;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        int i = g + k * G;
        if (i < A.n) y[i] = row_dot(A, nz, x, i);
    }
}

// z = P .* r (Jacobi: opDiagonal multiply, ldiv = false)
template <class T>
__global__ void k_jacobi_apply(int n, const T* __restrict__ P, const T* __restrict__ r, T* z, const KScalars* S) {
    jacobi_apply_body<T>(grid_tiles(), n, P, r, z, S);
}

template <class T>
__global__ void k_copy(int n, const T* __restrict__ a, T* b, const KScalars* S) {
    copy_body<T>(grid_tiles(), n, a, b, S);
}

// ---- CG ----
// p = z; gamma = <r,z>; initial stopping tests
template <class T>
__global__ void k_cg_start(int n, const T* __restrict__ r, const T* __restrict__ z, T* p, KScalars* S,
                           double* part) {
    cg_start_body<T>(grid_tiles(), n, r, z, p, S, part);
}

// q = A p_k; pAp = <p_k,q>; zero-curvature test; alpha = gamma / pAp
template <class T>
__global__ void __launch_bounds__(RED_THREADS, 8) k_cg_spmv(CSRView A, const T* __restrict__ nz,
                                                         const T* __restrict__ z, T* P0, T* P1, T* q, KScalars* S,
                                                         double* part) {
    cg_spmv_body<T>(grid_tiles(), A, nz, z, P0, P1, q, S, part);
}

// x += alpha p_k; r -= alpha q; [Jacobi: z = P r; <r,z>; finalize]
template <class T>
__global__ void __launch_bounds__(RED_THREADS, sizeof(T) == 4 ? 4 : 8) k_cg_update(int n, T* x, const T* __restrict__ P0, const T* __restrict__ P1, T* r,
                            const T* __restrict__ q, T* z, const T* __restrict__ P, int jacobi_fused, KScalars* S,
                            double* part) {
    cg_update_body<T>(grid_tiles(), n, x, P0, P1, r, q, z, P, jacobi_fused, S, part);
}

// <r,z> + finalize when z came from a separate preconditioner apply
template <class T>
__global__ void k_cg_rz(int n, const T* __restrict__ r, const T* __restrict__ z, KScalars* S, double* part) {
    cg_rz_body<T>(grid_tiles(), n, r, z, S, part);
}

template <class T, int NT>
__global__ void __launch_bounds__(NT, persist_min_blocks(NT))
    k_cg_persist(CSRView A, const T* __restrict__ nz, const T* __restrict__ Pj, int jacobi, T* x, T* r, T* z, T* P0,
                 T* P1, KScalars* S, double* part, double* part2, unsigned int* bar, int* err, int max_iters,
                 int pf_kb) {
    cg_persist_body<T, NT>(grid_tiles(), A, nz, Pj, jacobi, x, r, z, P0, P1, S, part, part2, bar, err, max_iters,
                           pf_kb);
}

// one block per SM, every G-th tile (cg_persist_mt_body); q in dynamic
// shared memory
template <class T, int NT>
__global__ void __launch_bounds__(NT, 1)
    k_cg_persist_mt(CSRView A, const T* __restrict__ nz, const T* __restrict__ Pj, int jacobi, T* x, T* r, T* z,
                    T* P0, T* P1, KScalars* S, double* part, double* part2, unsigned int* bar, int* err,
                    int max_iters) {
    extern __shared__ __align__(16) unsigned char mt_smem[];
    cg_persist_mt_body<T, NT>(A, nz, Pj, jacobi, x, r, z, P0, P1, S, part, part2, bar, err, max_iters,
                              reinterpret_cast<T*>(mt_smem));
}

// the cluster form: the grid is one cluster, block b owns tile b
template <class T>
__global__ void __launch_bounds__(1024, 1)
    k_cg_persist_cl(CSRView A, const T* __restrict__ nz, const T* __restrict__ Pj, int jacobi, T* x, T* r, T* z,
                    T* P0, T* P1, KScalars* S, int max_iters) {
    const TileCtx tc{(int)blockIdx.x, (A.n + RED_TILE - 1) / RED_TILE};
    cg_persist_body<T, 1024, true>(tc, A, nz, Pj, jacobi, x, r, z, P0, P1, S, nullptr, nullptr, nullptr, nullptr,
                                   max_iters, 0);
}

// field = x + dx (warm start shift)
__global__ void k_finish(int n, const double* __restrict__ x, const double* __restrict__ dx, double* field) {
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) field[i] = x[i] + dx[i];
    }
}

// ---- BiCGSTAB ----
// p = r; rNorm = ||r||; next_rho = <c,r>; initial tests
template <class T>
__global__ void k_bicg_start(int n, const T* __restrict__ c, const T* __restrict__ r, T* p, KScalars* S,
                             double* part0, double* part1) {
    bicg_start_body<T>(grid_tiles(), n, c, r, p, S, part0, part1);
}

// alpha = rho / <c,v> (rho = next_rho; iteration counter advances)
template <class T>
__global__ void k_bicg_alpha(int n, const T* __restrict__ c, const T* __restrict__ v, KScalars* S, double* part) {
    bicg_alpha_body<T>(grid_tiles(), n, c, v, S, part);
}

// s = r - alpha v; x = x + alpha p
template <class T>
__global__ void k_bicg_s(int n, const T* __restrict__ r, const T* __restrict__ v, const T* __restrict__ p, T* s,
                         T* x, const KScalars* S) {
    bicg_s_body<T>(grid_tiles(), n, r, v, p, s, x, S);
}

// omega = <t,s> / <t,t>
template <class T>
__global__ void k_bicg_omega(int n, const T* __restrict__ t, const T* __restrict__ s, KScalars* S, double* part0,
                             double* part1) {
    bicg_omega_body<T>(grid_tiles(), n, t, s, S, part0, part1);
}

// x = x + omega s; r = s - omega t; next_rho = <c,r>; ||r||; stopping tests
template <class T>
__global__ void k_bicg_xr(int n, T* x, const T* __restrict__ s, const T* __restrict__ t, T* r,
                          const T* __restrict__ c, KScalars* S, double* part0, double* part1) {
    bicg_xr_body<T>(grid_tiles(), n, x, s, t, r, c, S, part0, part1);
}

// p = r + beta (p - omega v)
template <class T>
__global__ void k_bicg_p(int n, const T* __restrict__ r, const T* __restrict__ v, T* p, const KScalars* S) {
    bicg_p_body<T>(grid_tiles(), n, r, v, p, S);
}

// multiply_row of the weighted Jacobi smoother (Smoothers_jacobi.jl:112-131):
// the row sum in storage order, less the diagonal term, then
// omega (1/a_ii) (b_i - sum) + (1 - omega) x_i into xt
__global__ void k_jacobi_smooth(CSRView A, const double* __restrict__ nz, const double* __restrict__ b,
                                const double* __restrict__ x, double* xt, double omega) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    double sum = row_dot(A, nz, x, i);
    const double a_ii = nz[A.diag[i]];
    const double xi = x[i];
    sum = sum - a_ii * xi;
    const double rD = 1.0 / a_ii;
    xt[i] = omega * rD * (b[i] - sum) + (1.0 - omega) * xi;
}

// ---- preconditioners ----
// update_Jacobi! (preconditioners_2_functions.jl:86-98)
__global__ void k_jacobi_update(CSRView A, const double* __restrict__ nz, double* P) {
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < A.n) {
            double d = fabs(nz[A.diag[i]]);
            P[i] = 1.0 / d;
        }
    }
}

// update_dilu_diagonal! restated per row (preconditioners_1_DILU.jl:43-82):
// D_i = A_ii - sum_{j<i, ascending} (A_ji A_ij) / D_j, one dependency level
__global__ void k_dilu_D(const int* __restrict__ rows, int nrows, CSRView A, const double* __restrict__ nz,
                         double* D) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows) return;
    dilu_D_row(A, nz, D, rows[t]);
}

// update_dilu_diagonal! for the row at level position k, reading the
// level-ordered lower triangle (coalesced over consecutive positions): the
// same operands, in the same order, as dilu_D_row.  Dr: where earlier
// levels' D values are read; the row's value goes to D (and Ds when given)
__device__ __forceinline__ void dilu_D_pos(const LevelDView& L, int k, const double* __restrict__ nz,
                                           const double* Dr, double* D, double* Ds) {
    const int i = L.rows[k];
    const int c = L.cnt[k];
    const int base = L.slice[k / SELL_C] + (k % SELL_C);
    int e[8];
#pragma unroll
    for (int m = 0; m < 8; ++m)
        if (m < c) e[m] = base + SELL_C * m;
    double d = nz[L.dslot[k]];
#pragma unroll
    for (int m = 0; m < 8; ++m)
        if (m < c) d = d - (nz[ld_stream(L.tsrc + e[m])] * nz[ld_stream(L.src + e[m])]) / Dr[ld_stream(L.col + e[m])];
    for (int m = 8; m < c; ++m) {
        const int em = base + SELL_C * m;
        d = d - (nz[ld_stream(L.tsrc + em)] * nz[ld_stream(L.src + em)]) / Dr[ld_stream(L.col + em)];
    }
    D[i] = d;
    if (Ds) Ds[i] = d;
}

// the D factor of a small system in one block, level by level over the
// level-ordered lower triangle; D in shared memory (smem) when it fits,
// copied out at the end
__global__ void __launch_bounds__(DILU_BLOCK_THREADS) k_dilu_D_lv_block(int n, LevelDView L,
                                                                        const double* __restrict__ nz, double* D,
                                                                        int smem) {
    extern __shared__ __align__(16) unsigned char dilu_smem[];
    double* Ds = smem ? reinterpret_cast<double*>(dilu_smem) : nullptr;
    for (int l = 0; l < L.nlev; ++l) {
        for (int k = L.off[l] + threadIdx.x; k < L.off[l + 1]; k += blockDim.x)
            dilu_D_pos(L, k, nz, smem ? (const double*)Ds : (const double*)D, D, Ds);
        __syncthreads();
    }
}

// the D factor of a small system in one block, level by level
__global__ void __launch_bounds__(DILU_BLOCK_THREADS) k_dilu_D_block(const int* __restrict__ rows,
                                                                     const int* __restrict__ off, int nlev,
                                                                     CSRView A, const double* __restrict__ nz,
                                                                     double* D) {
    for (int l = 0; l < nlev; ++l) {
        for (int k = off[l] + threadIdx.x; k < off[l + 1]; k += blockDim.x) dilu_D_row(A, nz, D, rows[k]);
        __syncthreads();
    }
}

// a whole DILU application (forward + backward sweeps) of a small system in one block
template <class T>
__global__ void __launch_bounds__(DILU_BLOCK_THREADS) k_dilu_block(int n, LevelView<T> lo, LevelView<T> up,
                                                                   const T* __restrict__ D, const T* __restrict__ b,
                                                                   T* y, int smem, const KScalars* S) {
    extern __shared__ __align__(16) unsigned char dilu_smem[];
    if (S && S->done) return;
    dilu_level_sweep<T>(n, lo, up, D, b, y, smem ? reinterpret_cast<T*>(dilu_smem) : y);
}

// One row of a level-ordered triangle with its first U slots in registers
// (column, value and, for the lower triangle, 1/D of the column): what a
// row's sweep reads that no sweep writes, so it can be loaded early.
template <class T, int U>
struct LvRow {
    int i, c, base;
    T rhs;
    int cj[U];
    T vj[U], dj[U];
};
template <class T, int U>
__device__ __forceinline__ void lv_load(const LevelView<T>& L, bool lower, int k, const T* __restrict__ D,
                                        const T* __restrict__ b, LvRow<T, U>& r) {
    r.i = L.rows[k];
    r.c = L.cnt[k];
    r.base = L.slice[k / SELL_C] + (k % SELL_C);
    r.rhs = lower ? b[r.i] : D[r.i];
#pragma unroll
    for (int j = 0; j < U; ++j)
        if (j < r.c) {
            const int e = r.base + SELL_C * j;
            r.cj[j] = ld_stream(L.col + e);
            r.vj[j] = ld_stream(L.val + e);
            if (lower) r.dj[j] = ld_stream(L.dinv + e);
        }
}
// the row's sweep: dilu_level_s's arithmetic (the same sum in the same
// entry order), slots past the first U read here
template <class T, bool LOWER, int U>
__device__ __forceinline__ void lv_apply(const LevelView<T>& L, const LvRow<T, U>& r, T* ys) {
    T sum = T(0);
#pragma unroll
    for (int j = 0; j < U; ++j)
        if (j < r.c) sum = LOWER ? sum + (r.vj[j] * ys[r.cj[j]]) * r.dj[j] : sum + r.vj[j] * ys[r.cj[j]];
    for (int j = U; j < r.c; ++j) {
        const int e = r.base + SELL_C * j;
        sum = LOWER ? sum + (ld_stream(L.val + e) * ys[ld_stream(L.col + e)]) * ld_stream(L.dinv + e)
                    : sum + ld_stream(L.val + e) * ys[ld_stream(L.col + e)];
    }
    ys[r.i] = LOWER ? r.rhs - sum : (ys[r.i] - sum) / r.rhs;
}

// Every level of one DILU application in one cooperative launch: the
// forward sweep's levels, then the backward sweep's, each spread over the
// whole grid (rows of a level are independent), with the bounded grid
// barrier between consecutive levels.  FP32: a thread loads its first row
// of the next level (indices, slots, right-hand side: nothing the sweep
// writes) before it enters the barrier, so only the gathers of y wait
// behind it (FP64 rows hold twice the registers; there the level runs as
// dilu_level_s, which measured faster).  Each row's arithmetic is that of
// the level kernels (dilu_level_s), bit for bit; only the launches go.  A
// barrier that gives up sets *err and ends every block.
constexpr int DILU_GRID_THREADS = 512;
template <class T>
__global__ void __launch_bounds__(DILU_GRID_THREADS, sizeof(T) == 4 ? 2 : 1) k_dilu_grid(LevelView<T> lo,
                                                                                       LevelView<T> up,
                                                                    const T* __restrict__ D,
                                                                    const T* __restrict__ b, T* y,
                                                                    unsigned int* bar, int* err,
                                                                    const KScalars* S) {
    constexpr int U = sizeof(T) == 4 ? 6 : 4;
    __shared__ int sh_err;
    if (S && S->done) return;
    const int start = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    const int total = lo.nlev + up.nlev;
    unsigned int nb = 0;
    if constexpr (sizeof(T) == 8) {
        for (int l = 0; l < total; ++l) {
            if (l < lo.nlev) {
                dilu_level_s<T, true>(lo, lo.off[l], lo.off[l + 1], D, b, y, start, stride);
            } else {
                const int u = l - lo.nlev;
                dilu_level_s<T, false>(up, up.off[u], up.off[u + 1], D, b, y, start, stride);
            }
            if (l + 1 < total && !grid_barrier(bar, gridDim.x, nb, err, &sh_err)) return;
        }
        return;
    }
    LvRow<T, U> r;
    bool have = false;  // r holds this thread's first row of level l
    if (total > 0 && lo.nlev > 0 && lo.off[0] + start < lo.off[1]) {
        lv_load<T, U>(lo, true, lo.off[0] + start, D, b, r);
        have = true;
    }
    for (int l = 0; l < total; ++l) {
        const bool lower = l < lo.nlev;
        const LevelView<T>& L = lower ? lo : up;
        const int lv = lower ? l : l - lo.nlev;
        const int k1 = L.off[lv + 1];
        int k = L.off[lv] + start;
        if (have) {
            if (lower)
                lv_apply<T, true, U>(L, r, y);
            else
                lv_apply<T, false, U>(L, r, y);
            k += stride;
        }
        for (; k < k1; k += stride) {
            lv_load<T, U>(L, lower, k, D, b, r);
            if (lower)
                lv_apply<T, true, U>(L, r, y);
            else
                lv_apply<T, false, U>(L, r, y);
        }
        if (l + 1 == total) break;
        const bool nlower = l + 1 < lo.nlev;
        const LevelView<T>& N = nlower ? lo : up;
        const int nv = nlower ? l + 1 : l + 1 - lo.nlev;
        have = N.off[nv] + start < N.off[nv + 1];
        if (have) lv_load<T, U>(N, nlower, N.off[nv] + start, D, b, r);
        if (!grid_barrier(bar, gridDim.x, nb, err, &sh_err)) return;
    }
}

// The DILU factor D of a large system in one cooperative launch: the lower
// triangle's levels spread over the grid, a grid barrier between levels,
// each row's arithmetic that of k_dilu_D (dilu_D_row).
__global__ void __launch_bounds__(DILU_GRID_THREADS) k_dilu_D_grid(const int* __restrict__ rows,
                                                                   const int* __restrict__ off, int nlev, CSRView A,
                                                                   const double* __restrict__ nz, double* D,
                                                                   unsigned int* bar, int* err) {
    __shared__ int sh_err;
    const int start = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    unsigned int nb = 0;
    for (int l = 0; l < nlev; ++l) {
        for (int k = off[l] + start; k < off[l + 1]; k += stride) dilu_D_row(A, nz, D, rows[k]);
        if (l + 1 < nlev && !grid_barrier(bar, gridDim.x, nb, err, &sh_err)) return;
    }
}

// the same over the level-ordered lower triangle
__global__ void __launch_bounds__(DILU_GRID_THREADS) k_dilu_D_lv_grid(LevelDView L, const double* __restrict__ nz,
                                                                      double* D, unsigned int* bar, int* err) {
    __shared__ int sh_err;
    const int start = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    unsigned int nb = 0;
    for (int l = 0; l < L.nlev; ++l) {
        for (int k = L.off[l] + start; k < L.off[l + 1]; k += stride) dilu_D_pos(L, k, nz, D, D, nullptr);
        if (l + 1 < L.nlev && !grid_barrier(bar, gridDim.x, nb, err, &sh_err)) return;
    }
}

// dinv[e] = T(1) / D[col[e]] (the forward sweep's per-entry reciprocal)
template <class T>
__global__ void k_level_dinv(long n, const int* __restrict__ col, const T* __restrict__ D, T* dinv) {
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
        dinv[e] = T(1) / D[ld_stream(col + e)];
}

// forward_substitution! (preconditioners_1_DILU.jl:84-98), one level
template <class T>
__global__ void k_dilu_fwd(const int* __restrict__ rows, int nrows, CSRView A, const T* __restrict__ nz,
                           const T* __restrict__ D, const T* __restrict__ b, T* y, const KScalars* S) {
    if (S && S->done) return;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows) return;
    dilu_fwd_row(A, nz, D, b, y, rows[t]);
}

// backward_substitution! (preconditioners_1_DILU.jl:100-114), one level, in place
template <class T>
__global__ void k_dilu_bwd(const int* __restrict__ rows, int nrows, CSRView A, const T* __restrict__ nz,
                           const T* __restrict__ D, T* x, const KScalars* S) {
    if (S && S->done) return;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows) return;
    dilu_bwd_row(A, nz, D, x, rows[t]);
}

// DILU sweeps over the level-ordered triangles: thread per position k of a
// level (row rows[k]); the entries are the row's own, in the row's order, so
// each row's sum is dilu_fwd_row's / dilu_bwd_row's
template <class T>
__global__ void k_dilu_fwd_lv(int k0, int k1, const int* __restrict__ rows, const int* __restrict__ slice,
                              const unsigned char* __restrict__ cnt, const int* __restrict__ col,
                              const T* __restrict__ val, const T* __restrict__ dinv, const T* __restrict__ b,
                              T* y, const KScalars* S) {
    if (S && S->done) return;
    const int k = k0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= k1) return;
    const int i = rows[k];
    const int base = slice[k / SELL_C] + (k % SELL_C), c = cnt[k];
    T sum = T(0);
    for (int j = 0; j < c; ++j) {
        const int e = base + SELL_C * j;
        sum = sum + (ld_stream(val + e) * y[ld_stream(col + e)]) * ld_stream(dinv + e);
    }
    y[i] = b[i] - sum;
}

template <class T>
__global__ void k_dilu_bwd_lv(int k0, int k1, const int* __restrict__ rows, const int* __restrict__ slice,
                              const unsigned char* __restrict__ cnt, const int* __restrict__ col,
                              const T* __restrict__ val, const T* __restrict__ D, T* x, const KScalars* S) {
    if (S && S->done) return;
    const int k = k0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= k1) return;
    const int i = rows[k];
    const int base = slice[k / SELL_C] + (k % SELL_C), c = cnt[k];
    T sum = T(0);
    for (int j = 0; j < c; ++j) {
        const int e = base + SELL_C * j;
        sum = sum + ld_stream(val + e) * x[ld_stream(col + e)];
    }
    x[i] = (x[i] - sum) / D[i];
}

// dst[e] = src_vals[src[e]] (refresh of a level-ordered triangle)
template <class T>
__global__ void k_gather_vals(long n, const int* __restrict__ src, const T* __restrict__ vals, T* dst) {
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
        dst[e] = vals[ld_stream(src + e)];
}

// residual (src/Solve/Solve_1_api.jl:441-464): ||b - A x|| / max(||b||, 1 if tiny)
__global__ void __launch_bounds__(RED_THREADS, 8) k_residual(CSRView A, const double* __restrict__ nz,
                                                          const double* __restrict__ x, const double* __restrict__ b,
                                                          KScalars* S, double* part0, double* part1, double* out) {
    __shared__ double sm[8];
    double a0 = 0.0, a1 = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < A.n) {
            double fx = row_dot(A, nz, x, i);
            double bi = b[i];
            double d = bi - fx;
            a0 = a0 + d * d;
            a1 = a1 + bi * bi;
        }
    }
    double t0 = block_tree(a0, sm);
    double t1 = block_tree(a1, sm);
    if (threadIdx.x == 0) {
        part0[blockIdx.x] = t0;
        part1[blockIdx.x] = t1;
    }
    if (!last_block(&S->counter2)) return;
    double sR = reduce_partials(part0, gridDim.x, sm);
    double sb = reduce_partials(part1, gridDim.x, sm);
    if (threadIdx.x == 0) {
        double normb = sqrt(sb);
        double denom = normb > jl_eps(normb) ? normb : 1.0;
        double res = sqrt(sR) / denom;
        S->resid = res;
        S->normb = normb;
        if (out) *out = res;
    }
}

// ---------------------------------------------------------------------------
// device-driven solve control (graph mode: the loops are conditional WHILE
// nodes whose condition these single-thread kernels set)
// ---------------------------------------------------------------------------
// the host's per-solve setup of the scalar block, as a kernel
__global__ void k_ks_init(KScalars* S, double atol, double rtol, int itmax, int mixed, double inner_rtol) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    KScalars z = {};
    z.atol = atol;
    z.rtol = rtol;
    z.itmax = itmax;
    z.mixed = mixed;
    z.inner_rtol = inner_rtol;
    *S = z;
}

// end of a Krylov loop body: continue while the solve runs, at most `cap`
// bodies (a solve that has not finished by then is stopped as KS_LOOP_CAP);
// adds the body's kernel count to the launch counter
__global__ void k_loop_cond(cudaGraphConditionalHandle h, KScalars* S, int cap, int body_kernels,
                            unsigned long long* launches) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    atomicAdd(launches, (unsigned long long)body_kernels);
    S->loops = S->loops + 1;
    bool go = !S->done && S->loops < cap;
    if (!go && !S->done) {
        S->done = 1;
        S->status = KS_LOOP_CAP;
    }
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

// a WHILE loop is entered with its condition set to 1 by this kernel, placed
// right before the node (every execution of the enclosing graph or body)
__global__ void k_set_cond(cudaGraphConditionalHandle h, unsigned int v) {
    if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, v);
}

// start of a defect-correction step: the inner solve state is reset
__global__ void k_outer_prep(KScalars* S) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    S->iter = 0;
    S->done = 0;
    S->status = KS_RUNNING;
}

// field += inner solution unless the defect already met the target
__global__ void k_correct_masked(int n, double* field, const float* __restrict__ x, const KScalars* S) {
    if (S->outer_conv) return;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) field[i] = field[i] + (double)x[i];
    }
}

// end of a defect-correction step (the host loop's exit tests, on the device)
__global__ void k_outer_cond(cudaGraphConditionalHandle h, KScalars* S, int max_outer, int body_kernels,
                             unsigned long long* launches) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    atomicAdd(launches, (unsigned long long)body_kernels);
    bool stop = S->outer_conv != 0;
    if (!stop) {
        S->total = S->total + S->iter;
        int st = S->status;
        stop = st == KS_ZERO_CURV || st == KS_BREAKDOWN || st == KS_TIRED || st == KS_LOOP_CAP ||
               (st == KS_SOLVED && S->eps <= S->eps_outer);
    }
    S->outer = S->outer + 1;
    if (!stop && S->outer >= max_outer) stop = true;
    cudaGraphSetConditional(h, stop ? 0u : 1u);
}

// iterations and status of the finished solve into out[0..1]
__global__ void k_record(const KScalars* S, int* out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    out[0] = S->mixed ? S->total : S->iter;
    out[1] = S->status;
}

__global__ void k_coop_noop() {}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// capture (top level or inside a WHILE body) and run a no-op launched
// cooperatively (one block) or as one cluster of two blocks
static bool capture_probe(bool in_while, bool cluster) {
    cudaStream_t s = nullptr, s2 = nullptr;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster ? 2 : 1);
    cfg.blockDim = dim3(32);
    cudaLaunchAttribute at[1];
    if (cluster) {
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 2;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
    } else {
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
    }
    cfg.attrs = at;
    cfg.numAttrs = 1;
    void* noargs[1] = {nullptr};
    bool ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
        if (!in_while) {
            cfg.stream = s;
            ok = cudaLaunchKernelExC(&cfg, (const void*)k_coop_noop, noargs) == cudaSuccess;
        } else {
            // WHILE node entered with its condition at 1; the body runs the
            // no-op and sets the condition to 0, so it runs exactly once
            cudaStreamCaptureStatus cs;
            cudaGraph_t cg = nullptr;
            const cudaGraphNode_t* deps = nullptr;
            size_t nd = 0;
            cudaGraphConditionalHandle h;
            ok = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd) == cudaSuccess &&
                 cudaGraphConditionalHandleCreate(&h, cg, 1, cudaGraphCondAssignDefault) == cudaSuccess;
            cudaGraphNodeParams prm = {};
            cudaGraphNode_t node;
            if (ok) {
                prm.type = cudaGraphNodeTypeConditional;
                prm.conditional.handle = h;
                prm.conditional.type = cudaGraphCondTypeWhile;
                prm.conditional.size = 1;
                ok = cudaGraphAddNode(&node, cg, deps, nd, &prm) == cudaSuccess;
            }
            if (ok) ok = cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking) == cudaSuccess;
            if (ok)
                ok = cudaStreamBeginCaptureToGraph(s2, prm.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                cfg.stream = s2;
                bool l1 = cudaLaunchKernelExC(&cfg, (const void*)k_coop_noop, noargs) == cudaSuccess;
                k_set_cond<<<1, 32, 0, s2>>>(h, 0u);
                bool l2 = cudaGetLastError() == cudaSuccess;
                cudaGraph_t tmp = nullptr;
                bool l3 = cudaStreamEndCapture(s2, &tmp) == cudaSuccess;
                ok = l1 && l2 && l3;
            }
        }
        cudaError_t ee = cudaStreamEndCapture(s, &g);
        ok = ok && ee == cudaSuccess;
    }
    ok = ok && cudaGraphInstantiate(&ge, g, 0) == cudaSuccess;
    ok = ok && cudaGraphLaunch(ge, s) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    if (s2) cudaStreamDestroy(s2);
    if (s) cudaStreamDestroy(s);
    cudaGetLastError();
    return ok;
}

bool kr_coop_capture_ok(bool in_while) {
    static int state[2] = {-1, -1};
    int& st = state[in_while ? 1 : 0];
    if (st < 0) st = capture_probe(in_while, false) ? 1 : 0;
    return st == 1;
}

bool kr_cluster_capture_ok(bool in_while) {
    static int state[2] = {-1, -1};
    int& st = state[in_while ? 1 : 0];
    if (st < 0) st = capture_probe(in_while, true) ? 1 : 0;
    return st == 1;
}

static inline int tiles(int n) { return n <= 0 ? 1 : (n + RED_TILE - 1) / RED_TILE; }
#define TILE_LAUNCH(n) tiles(n), RED_THREADS, 0

void kr_init_resid(cudaStream_t s, const CSRView& A, const double* nz, const double* b, const double* field,
                   double* dx, double* x, double* r) {
    k_init_resid<<<TILE_LAUNCH(A.n), s>>>(A, nz, b, field, dx, x, r);
    XCAL_CHECK_LAUNCH();
}
void kr_defect(cudaStream_t s, const CSRView& A, const double* nz, const double* b, const double* field, float* d,
               float* x) {
    k_defect<<<TILE_LAUNCH(A.n), s>>>(A, nz, b, field, d, x);
    XCAL_CHECK_LAUNCH();
}
void kr_correct(cudaStream_t s, int n, double* field, const float* x) {
    k_correct<<<TILE_LAUNCH(n), s>>>(n, field, x);
    XCAL_CHECK_LAUNCH();
}
void kr_to_float(cudaStream_t s, long n, const double* src, float* dst) {
    if (n <= 0) return;
    long blocks = (n + 255) / 256;
    k_to_float<<<(int)(blocks < 148L * 16 ? blocks : 148L * 16), 256, 0, s>>>(n, src, dst);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_spmv(cudaStream_t s, const CSRView& A, const T* nz, const T* x, T* y, const KScalars* S) {
    k_spmv<T><<<TILE_LAUNCH(A.n), s>>>(A, nz, x, y, S);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_spmv_shaped(cudaStream_t s, const SpmvShape& sh, const CSRView& A, const T* nz, const T* x, T* y,
                    const KScalars* S) {
    if (sh.rows_per_thread <= 0) {
        kr_spmv(s, A, nz, x, y, S);
        return;
    }
    const long per_block = (long)sh.block * sh.rows_per_thread;
    const int grid = (int)((A.n + per_block - 1) / per_block);
    if (grid <= 0) return;
    switch (sh.rows_per_thread) {
        case 1: k_spmv_rows<T, 1><<<grid, sh.block, 0, s>>>(A, nz, x, y, S); break;
        case 2: k_spmv_rows<T, 2><<<grid, sh.block, 0, s>>>(A, nz, x, y, S); break;
        default: k_spmv_rows<T, 4><<<grid, sh.block, 0, s>>>(A, nz, x, y, S); break;
    }
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_jacobi_apply(cudaStream_t s, int n, const T* P, const T* r, T* z, const KScalars* S) {
    k_jacobi_apply<T><<<TILE_LAUNCH(n), s>>>(n, P, r, z, S);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_copy(cudaStream_t s, int n, const T* a, T* b, const KScalars* S) {
    k_copy<T><<<TILE_LAUNCH(n), s>>>(n, a, b, S);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_cg_start(cudaStream_t s, int n, const T* r, const T* z, T* p, KScalars* S, double* part) {
    k_cg_start<T><<<TILE_LAUNCH(n), s>>>(n, r, z, p, S, part);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_cg_spmv(cudaStream_t s, const CSRView& A, const T* nz, const T* z, T* P0, T* P1, T* q, KScalars* S,
                double* part) {
    k_cg_spmv<T><<<TILE_LAUNCH(A.n), s>>>(A, nz, z, P0, P1, q, S, part);
    XCAL_CHECK_LAUNCH();
}
static_assert(PERSIST_WIDTHS[2] == RED_THREADS, "narrow persistent form is one canonical tile row set per thread");

int persist_pick(PersistCaps& c, const void* const k[3], int ntiles, int width) {
    if (!c.init) {
        c.init = true;
        int dev = 0, sms = 0;
        bool okd = cudaGetDevice(&dev) == cudaSuccess &&
                   cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess;
        for (int w = 0; w < 3; ++w) {
            int per = 0;
            if (!okd || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k[w], PERSIST_WIDTHS[w], 0) != cudaSuccess) {
                cudaGetLastError();
                per = 0;
            }
            c.cap[w] = per * sms;
        }
    }
    if (ntiles <= 0) return -1;
    for (int w = 0; w < 3; ++w)
        if ((width == 0 || width == PERSIST_WIDTHS[w]) && ntiles <= c.cap[w]) return w;
    return -1;
}

bool persist_launch(PersistCaps& c, int w, const void* kernel, int ntiles, cudaStream_t s, void** args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ntiles);
    cfg.blockDim = dim3(PERSIST_WIDTHS[w]);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelExC(&cfg, kernel, args);
    if (e == cudaErrorCooperativeLaunchTooLarge) {
        cudaGetLastError();
        c.cap[w] = ntiles - 1;
        return false;
    }
    XCAL_CUDA(e);
    XCAL_CHECK_LAUNCH();
    return true;
}

int persist_cluster_size(const void* kernel, int tiles) {
    if (tiles <= 0 || tiles > PERSIST_CLUSTER_MAX) return 0;
    int C = 1;
    while (C < tiles) C *= 2;
    // schedulability per (kernel, C), found once
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, bool> ok;
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_pair(kernel, C);
    auto it = ok.find(key);
    if (it == ok.end()) {
        bool good = true;
        if (C > 8)
            good = cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess;
        int num = 0;
        if (good) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(C);
            cfg.blockDim = dim3(1024);
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = C;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            good = cudaOccupancyMaxActiveClusters(&num, kernel, &cfg) == cudaSuccess && num >= 1;
        }
        cudaGetLastError();
        it = ok.emplace(key, good).first;
    }
    return it->second ? C : 0;
}

void persist_cluster_launch(const void* kernel, int C, int nclusters, cudaStream_t s, void** args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C * nclusters);
    cfg.blockDim = dim3(1024);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    XCAL_CUDA(cudaLaunchKernelExC(&cfg, kernel, args));
    XCAL_CHECK_LAUNCH();
}

template <class T>
bool kr_cg_persist(cudaStream_t s, const CSRView& A, const T* nz, const T* P, int jacobi, T* x, T* r, T* z, T* P0,
                   T* P1, KScalars* S, double* part, double* part2, unsigned int* bar, int* err, int max_iters,
                   int width, int pf_kb, bool reset_err) {
    static PersistCaps caps;  // co-resident blocks per width (per process, one device type)
    static const void* const kern[3] = {(const void*)k_cg_persist<T, 1024>, (const void*)k_cg_persist<T, 512>,
                                        (const void*)k_cg_persist<T, RED_THREADS>};
    const int nt = tiles(A.n);
    // the automatic choice past the one-tile-per-block forms: one block per
    // SM owning up to three tiles (measured on B200, FP64: 42.1 against 47.1
    // us per iteration at 432 tiles; at 1,024 tiles the narrow form is
    // faster, 73.0 against 100.3 us)
    if (width == 0 || width == PERSIST_COOP_ONLY) {
        static int sms_auto = -1;
        if (sms_auto < 0) {
            int dev = 0;
            if (cudaGetDevice(&dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&sms_auto, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
                sms_auto = 0;
            cudaGetLastError();
        }
        if (sms_auto > 0 && nt > 2 * sms_auto && nt <= 3 * sms_auto &&
            kr_cg_persist(s, A, nz, P, jacobi, x, r, z, P0, P1, S, part, part2, bar, err, max_iters, PERSIST_MT1024,
                          pf_kb, reset_err))
            return true;
    }
    if (width == PERSIST_MT1024 || width == PERSIST_MT512) {
        // one block per SM (fewer when there are fewer tiles), the tiles
        // dealt round robin; false when q of a block's tiles does not fit
        static int sms = -1, ok_attr[2] = {-1, -1};
        const int f = width == PERSIST_MT1024 ? 0 : 1;
        const void* km = f == 0 ? (const void*)k_cg_persist_mt<T, 1024> : (const void*)k_cg_persist_mt<T, 512>;
        if (sms < 0) {
            int dev = 0;
            if (cudaGetDevice(&dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
                sms = 0;
            cudaGetLastError();
        }
        if (ok_attr[f] < 0) {
            int per = 0;
            ok_attr[f] = cudaFuncSetAttribute(km, cudaFuncAttributeMaxDynamicSharedMemorySize, PERSIST_MT_SMEM) ==
                                 cudaSuccess &&
                         cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, km, f == 0 ? 1024 : 512,
                                                                       PERSIST_MT_SMEM) == cudaSuccess &&
                         per >= 1;
            cudaGetLastError();
        }
        if (sms <= 0 || ok_attr[f] != 1 || nt <= 0) return false;
        const int G = std::min(sms, nt);
        const int tpb = (nt + G - 1) / G;
        const size_t smem = (size_t)tpb * RED_TILE * sizeof(T);
        if (smem > (size_t)PERSIST_MT_SMEM) return false;
        XCAL_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned int), s));
        if (reset_err) XCAL_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
        CSRView Av = A;
        void* args[] = {&Av, (void*)&nz, (void*)&P, &jacobi, &x,   &r,   &z,
                        &P0, &P1,        &S,        &part,   &part2, &bar, &err, &max_iters};
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(G);
        cfg.blockDim = dim3(f == 0 ? 1024 : 512);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        XCAL_CUDA(cudaLaunchKernelExC(&cfg, km, args));
        XCAL_CHECK_LAUNCH();
        return true;
    }
    if (width == 0 || width == PERSIST_CLUSTER_ONLY) {
        const void* kc = (const void*)k_cg_persist_cl<T>;
        const int C = persist_cluster_size(kc, nt);
        if (C > 0) {
            CSRView Av = A;
            void* args[] = {&Av, (void*)&nz, (void*)&P, &jacobi, &x, &r, &z, &P0, &P1, &S, &max_iters};
            persist_cluster_launch(kc, C, 1, s, args);
            return true;
        }
        if (width == PERSIST_CLUSTER_ONLY) return false;
    }
    const int w = persist_pick(caps, kern, nt, width == PERSIST_COOP_ONLY ? 0 : width);
    if (w < 0) return false;
    XCAL_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned int), s));
    if (reset_err) XCAL_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    CSRView Av = A;
    void* args[] = {&Av, (void*)&nz, (void*)&P, &jacobi, &x,         &r,    &z,
                    &P0, &P1,        &S,        &part,   &part2,     &bar,  &err,
                    &max_iters, &pf_kb};
    return persist_launch(caps, w, kern[w], nt, s, args);
}
template <class T>
void kr_cg_update(cudaStream_t s, int n, T* x, const T* P0, const T* P1, T* r, const T* q, T* z, const T* P,
                  int jacobi_fused, KScalars* S, double* part) {
    k_cg_update<T><<<TILE_LAUNCH(n), s>>>(n, x, P0, P1, r, q, z, P, jacobi_fused, S, part);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_cg_rz(cudaStream_t s, int n, const T* r, const T* z, KScalars* S, double* part) {
    k_cg_rz<T><<<TILE_LAUNCH(n), s>>>(n, r, z, S, part);
    XCAL_CHECK_LAUNCH();
}
void kr_finish(cudaStream_t s, int n, const double* x, const double* dx, double* field) {
    k_finish<<<TILE_LAUNCH(n), s>>>(n, x, dx, field);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_bicg_start(cudaStream_t s, int n, const T* c, const T* r, T* p, KScalars* S, double* part0,
                   double* part1) {
    k_bicg_start<T><<<TILE_LAUNCH(n), s>>>(n, c, r, p, S, part0, part1);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_bicg_alpha(cudaStream_t s, int n, const T* c, const T* v, KScalars* S, double* part) {
    k_bicg_alpha<T><<<TILE_LAUNCH(n), s>>>(n, c, v, S, part);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_bicg_s(cudaStream_t s_, int n, const T* r, const T* v, const T* p, T* s, T* x, const KScalars* S) {
    k_bicg_s<T><<<TILE_LAUNCH(n), s_>>>(n, r, v, p, s, x, S);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_bicg_omega(cudaStream_t s_, int n, const T* t, const T* s, KScalars* S, double* part0, double* part1) {
    k_bicg_omega<T><<<TILE_LAUNCH(n), s_>>>(n, t, s, S, part0, part1);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_bicg_xr(cudaStream_t s_, int n, T* x, const T* s, const T* t, T* r, const T* c, KScalars* S,
                double* part0, double* part1) {
    k_bicg_xr<T><<<TILE_LAUNCH(n), s_>>>(n, x, s, t, r, c, S, part0, part1);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_bicg_p(cudaStream_t s, int n, const T* r, const T* v, T* p, const KScalars* S) {
    k_bicg_p<T><<<TILE_LAUNCH(n), s>>>(n, r, v, p, S);
    XCAL_CHECK_LAUNCH();
}
void kr_jacobi_smooth(cudaStream_t s, const CSRView& A, const double* nz, const double* b, double* x, double* xt,
                      int loops, double omega) {
    for (int l = 0; l < loops; ++l) {
        k_jacobi_smooth<<<(A.n + 255) / 256, 256, 0, s>>>(A, nz, b, x, xt, omega);
        XCAL_CHECK_LAUNCH();
        XCAL_CUDA(cudaMemcpyAsync(x, xt, (size_t)A.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
}
void kr_jacobi_update(cudaStream_t s, const CSRView& A, const double* nz, double* P) {
    k_jacobi_update<<<TILE_LAUNCH(A.n), s>>>(A, nz, P);
    XCAL_CHECK_LAUNCH();
}
void kr_dilu_D(cudaStream_t s, const int* rows, int nrows, const CSRView& A, const double* nz, double* D) {
    if (nrows <= 0) return;
    k_dilu_D<<<(nrows + 255) / 256, 256, 0, s>>>(rows, nrows, A, nz, D);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_dilu_fwd(cudaStream_t s, const int* rows, int nrows, const CSRView& A, const T* nz, const T* D, const T* b,
                 T* y, const KScalars* S) {
    if (nrows <= 0) return;
    k_dilu_fwd<T><<<(nrows + 255) / 256, 256, 0, s>>>(rows, nrows, A, nz, D, b, y, S);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_dilu_bwd(cudaStream_t s, const int* rows, int nrows, const CSRView& A, const T* nz, const T* D, T* x,
                 const KScalars* S) {
    if (nrows <= 0) return;
    k_dilu_bwd<T><<<(nrows + 255) / 256, 256, 0, s>>>(rows, nrows, A, nz, D, x, S);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_dilu_fwd_lv(cudaStream_t s, int k0, int k1, const int* rows, const int* slice, const unsigned char* cnt,
                    const int* col, const T* val, const T* dinv, const T* b, T* y, const KScalars* S) {
    if (k1 <= k0) return;
    k_dilu_fwd_lv<T><<<(k1 - k0 + 255) / 256, 256, 0, s>>>(k0, k1, rows, slice, cnt, col, val, dinv, b, y, S);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_level_dinv(cudaStream_t s, long nslots, const int* col, const T* D, T* dinv) {
    if (nslots <= 0) return;
    const long blocks = std::min((nslots + 255) / 256, 148L * 16);
    k_level_dinv<T><<<(int)blocks, 256, 0, s>>>(nslots, col, D, dinv);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_dilu_bwd_lv(cudaStream_t s, int k0, int k1, const int* rows, const int* slice, const unsigned char* cnt,
                    const int* col, const T* val, const T* D, T* x, const KScalars* S) {
    if (k1 <= k0) return;
    k_dilu_bwd_lv<T><<<(k1 - k0 + 255) / 256, 256, 0, s>>>(k0, k1, rows, slice, cnt, col, val, D, x, S);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_gather_vals(cudaStream_t s, long n, const int* src, const T* vals, T* dst) {
    if (n <= 0) return;
    long blocks = (n + 255) / 256;
    k_gather_vals<T><<<(int)(blocks < 148L * 16 ? blocks : 148L * 16), 256, 0, s>>>(n, src, vals, dst);
    XCAL_CHECK_LAUNCH();
}
void kr_dilu_D_lv_block(cudaStream_t s, int n, const LevelDView& L, const double* nz, double* D) {
    if (L.nlev <= 0) return;
    static bool attr_set = false;
    if (!attr_set) {
        XCAL_CUDA(cudaFuncSetAttribute((const void*)k_dilu_D_lv_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       DILU_SMEM_MAX_BYTES));
        attr_set = true;
    }
    const size_t bytes = (size_t)n * sizeof(double);
    const int smem = bytes <= (size_t)DILU_SMEM_MAX_BYTES ? 1 : 0;
    k_dilu_D_lv_block<<<1, DILU_BLOCK_THREADS, smem ? bytes : 0, s>>>(n, L, nz, D, smem);
    XCAL_CHECK_LAUNCH();
}
bool kr_dilu_D_lv_grid(cudaStream_t s, const LevelDView& L, const double* nz, double* D, unsigned int* bar,
                       int* err) {
    static int blocks = -1;
    if (blocks < 0) {
        int dev = 0, sms = 0, per = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)k_dilu_D_lv_grid, DILU_GRID_THREADS,
                                                          0) == cudaSuccess)
            blocks = sms * std::min(per, 2);
        else
            blocks = 0;
        cudaGetLastError();
    }
    if (blocks <= 0 || L.nlev <= 0) return false;
    XCAL_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned int), s));
    LevelDView Lv = L;
    void* args[] = {&Lv, (void*)&nz, &D, &bar, &err};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(DILU_GRID_THREADS);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    XCAL_CUDA(cudaLaunchKernelExC(&cfg, (const void*)k_dilu_D_lv_grid, args));
    XCAL_CHECK_LAUNCH();
    return true;
}
void kr_dilu_D_block(cudaStream_t s, const int* rows, const int* off, int nlev, const CSRView& A, const double* nz,
                     double* D) {
    if (nlev <= 0) return;
    k_dilu_D_block<<<1, DILU_BLOCK_THREADS, 0, s>>>(rows, off, nlev, A, nz, D);
    XCAL_CHECK_LAUNCH();
}
template <class T>
void kr_dilu_block(cudaStream_t s, int n, const LevelView<T>& lo, const LevelView<T>& up, const T* D, const T* b,
                   T* y, const KScalars* S) {
    static bool attr_set = false;  // shared-memory limit of the kernel (per process, one device type)
    if (!attr_set) {
        XCAL_CUDA(cudaFuncSetAttribute(k_dilu_block<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       DILU_SMEM_MAX_BYTES));
        attr_set = true;
    }
    const size_t bytes = (size_t)n * sizeof(T);
    const int smem = bytes <= (size_t)DILU_SMEM_MAX_BYTES ? 1 : 0;
    k_dilu_block<T><<<1, DILU_BLOCK_THREADS, smem ? bytes : 0, s>>>(n, lo, up, D, b, y, smem, S);
    XCAL_CHECK_LAUNCH();
}
template <class T>
bool kr_dilu_grid(cudaStream_t s, const LevelView<T>& lo, const LevelView<T>& up, const T* D, const T* b, T* y,
                  unsigned int* bar, int* err, const KScalars* S) {
    // blocks: up to two per SM that are co-resident (found once per process
    // and value type); 0 = the device cannot run it cooperatively
    static int blocks = -1;
    if (blocks < 0) {
        int dev = 0, sms = 0, per = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)k_dilu_grid<T>, DILU_GRID_THREADS, 0) ==
                cudaSuccess)
            blocks = sms * std::min(per, 2);
        else
            blocks = 0;
        cudaGetLastError();
    }
    if (blocks <= 0) return false;
    XCAL_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned int), s));
    LevelView<T> l = lo, u = up;
    void* args[] = {&l, &u, (void*)&D, (void*)&b, &y, &bar, &err, (void*)&S};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(DILU_GRID_THREADS);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    XCAL_CUDA(cudaLaunchKernelExC(&cfg, (const void*)k_dilu_grid<T>, args));
    XCAL_CHECK_LAUNCH();
    return true;
}
bool kr_dilu_D_grid(cudaStream_t s, const int* rows, const int* off, int nlev, const CSRView& A, const double* nz,
                    double* D, unsigned int* bar, int* err) {
    static int blocks = -1;
    if (blocks < 0) {
        int dev = 0, sms = 0, per = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)k_dilu_D_grid, DILU_GRID_THREADS, 0) ==
                cudaSuccess)
            blocks = sms * std::min(per, 2);
        else
            blocks = 0;
        cudaGetLastError();
    }
    if (blocks <= 0 || nlev <= 0) return false;
    XCAL_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned int), s));
    CSRView Av = A;
    void* args[] = {(void*)&rows, (void*)&off, &nlev, &Av, (void*)&nz, &D, &bar, &err};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(DILU_GRID_THREADS);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    XCAL_CUDA(cudaLaunchKernelExC(&cfg, (const void*)k_dilu_D_grid, args));
    XCAL_CHECK_LAUNCH();
    return true;
}
template bool kr_dilu_grid<double>(cudaStream_t, const LevelView<double>&, const LevelView<double>&, const double*,
                                   const double*, double*, unsigned int*, int*, const KScalars*);
template bool kr_dilu_grid<float>(cudaStream_t, const LevelView<float>&, const LevelView<float>&, const float*,
                                  const float*, float*, unsigned int*, int*, const KScalars*);

void kr_residual(cudaStream_t s, const CSRView& A, const double* nz, const double* x, const double* b, KScalars* S,
                 double* part0, double* part1, double* out) {
    k_residual<<<TILE_LAUNCH(A.n), s>>>(A, nz, x, b, S, part0, part1, out);
    XCAL_CHECK_LAUNCH();
}

void kr_ks_init(cudaStream_t s, KScalars* S, double atol, double rtol, int itmax, int mixed, double inner_rtol) {
    k_ks_init<<<1, 32, 0, s>>>(S, atol, rtol, itmax, mixed, inner_rtol);
    XCAL_CHECK_LAUNCH();
}
void kr_loop_cond(cudaStream_t s, cudaGraphConditionalHandle h, KScalars* S, int cap, int body_kernels,
                  unsigned long long* launches) {
    k_loop_cond<<<1, 32, 0, s>>>(h, S, cap, body_kernels, launches);
    XCAL_CHECK_LAUNCH();
}
void kr_set_cond(cudaStream_t s, cudaGraphConditionalHandle h, unsigned int v) {
    k_set_cond<<<1, 32, 0, s>>>(h, v);
    XCAL_CHECK_LAUNCH();
}
void kr_outer_prep(cudaStream_t s, KScalars* S) {
    k_outer_prep<<<1, 32, 0, s>>>(S);
    XCAL_CHECK_LAUNCH();
}
void kr_correct_masked(cudaStream_t s, int n, double* field, const float* x, const KScalars* S) {
    k_correct_masked<<<TILE_LAUNCH(n), s>>>(n, field, x, S);
    XCAL_CHECK_LAUNCH();
}
void kr_outer_cond(cudaStream_t s, cudaGraphConditionalHandle h, KScalars* S, int max_outer, int body_kernels,
                   unsigned long long* launches) {
    k_outer_cond<<<1, 32, 0, s>>>(h, S, max_outer, body_kernels, launches);
    XCAL_CHECK_LAUNCH();
}
void kr_record(cudaStream_t s, const KScalars* S, int* out) {
    k_record<<<1, 32, 0, s>>>(S, out);
    XCAL_CHECK_LAUNCH();
}

// the two value types of the Krylov launchers
#define XCAL_KRYLOV_INSTANTIATE(T)                                                                              \
    template void kr_spmv<T>(cudaStream_t, const CSRView&, const T*, const T*, T*, const KScalars*);             \
    template void kr_spmv_shaped<T>(cudaStream_t, const SpmvShape&, const CSRView&, const T*, const T*, T*,      \
                                    const KScalars*);                                                           \
    template void kr_jacobi_apply<T>(cudaStream_t, int, const T*, const T*, T*, const KScalars*);                \
    template void kr_copy<T>(cudaStream_t, int, const T*, T*, const KScalars*);                                  \
    template void kr_cg_start<T>(cudaStream_t, int, const T*, const T*, T*, KScalars*, double*);                 \
    template void kr_cg_spmv<T>(cudaStream_t, const CSRView&, const T*, const T*, T*, T*, T*, KScalars*,         \
                                double*);                                                                       \
    template void kr_cg_update<T>(cudaStream_t, int, T*, const T*, const T*, T*, const T*, T*, const T*, int,    \
                                  KScalars*, double*);                                                          \
    template void kr_cg_rz<T>(cudaStream_t, int, const T*, const T*, KScalars*, double*);                        \
    template bool kr_cg_persist<T>(cudaStream_t, const CSRView&, const T*, const T*, int, T*, T*, T*, T*, T*,    \
                                   KScalars*, double*, double*, unsigned int*, int*, int, int, int, bool);      \
    template void kr_bicg_start<T>(cudaStream_t, int, const T*, const T*, T*, KScalars*, double*, double*);      \
    template void kr_bicg_alpha<T>(cudaStream_t, int, const T*, const T*, KScalars*, double*);                   \
    template void kr_bicg_s<T>(cudaStream_t, int, const T*, const T*, const T*, T*, T*, const KScalars*);        \
    template void kr_bicg_omega<T>(cudaStream_t, int, const T*, const T*, KScalars*, double*, double*);          \
    template void kr_bicg_xr<T>(cudaStream_t, int, T*, const T*, const T*, T*, const T*, KScalars*, double*,     \
                                double*);                                                                       \
    template void kr_bicg_p<T>(cudaStream_t, int, const T*, const T*, T*, const KScalars*);                      \
    template void kr_dilu_fwd<T>(cudaStream_t, const int*, int, const CSRView&, const T*, const T*, const T*, T*, \
                                 const KScalars*);                                                              \
    template void kr_dilu_bwd<T>(cudaStream_t, const int*, int, const CSRView&, const T*, const T*, T*,          \
                                 const KScalars*);                                                              \
    template void kr_dilu_block<T>(cudaStream_t, int, const LevelView<T>&, const LevelView<T>&, const T*,       \
                                   const T*, T*, const KScalars*);                                              \
    template void kr_level_dinv<T>(cudaStream_t, long, const int*, const T*, T*);                                \
    template void kr_dilu_fwd_lv<T>(cudaStream_t, int, int, const int*, const int*, const unsigned char*,         \
                                    const int*, const T*, const T*, const T*, T*, const KScalars*);             \
    template void kr_dilu_bwd_lv<T>(cudaStream_t, int, int, const int*, const int*, const unsigned char*,         \
                                    const int*, const T*, const T*, T*, const KScalars*);                       \
    template void kr_gather_vals<T>(cudaStream_t, long, const int*, const T*, T*);
XCAL_KRYLOV_INSTANTIATE(double)
XCAL_KRYLOV_INSTANTIATE(float)

}  // namespace xcal
