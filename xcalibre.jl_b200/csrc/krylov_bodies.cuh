// krylov_bodies.cuh -- per-tile bodies of the Krylov kernels.
//
// Each body works on one canonical tile `tc.tile` of a system with
// `tc.ntiles` tiles.  The single-system kernels (kernels_krylov.cu) pass the
// grid (tile = block, ntiles = grid size); the batched kernels
// (kernels_batch.cu) pass a (system, local tile) entry of their tile map, so a
// system's arithmetic -- row sums, reduction trees, scalar decisions -- is the
// same whether it is solved alone or inside a batch.
#pragma once
#include <cooperative_groups.h>

#include "dev_common.cuh"
#include "kernels.hpp"

namespace xcal {

template <class T>
__device__ __forceinline__ T row_dot(const CSRView& A, const T* __restrict__ nz, const T* __restrict__ x, int i) {
    // xmul! row (src/Multithread/spmvm.jl:47-53): sequential from 0.0
    T acc = T(0);
    const int rb = row_base(A, i), rl = A.len[i];
    for (int k = 0; k < rl; ++k) {
        int e = rb + SELL_C * k;
        acc = acc + ld_stream(nz + e) * x[ld_stream(A.colval + e)];
    }
    return acc;
}

// CG stopping decisions after gamma_next = <r,z> (Krylov.jl cg!)
__device__ __forceinline__ void cg_finalize(KScalars* S, double gamma_next) {
    double rNorm = sqrt(gamma_next);
    S->rNorm = rNorm;
    bool mach = (rNorm + 1.0 <= 1.0);
    bool solved = (rNorm <= S->eps) || mach;
    if (!solved) {
        double beta = gamma_next / S->gamma;
        S->pNorm2 = gamma_next + (beta * beta) * S->pNorm2;
        S->gamma = gamma_next;
        S->beta = beta;
    }
    S->iter = S->iter + 1;
    bool tired = S->iter >= S->itmax;
    if (solved) {
        S->done = 1;
        S->status = KS_SOLVED;
    } else if (tired) {
        S->done = 1;
        S->status = KS_TIRED;
    }
}

// Stopping tolerance at the start of a solve.  Plain mode: Krylov.jl's
// atol + rtol*||r0||.  Mixed mode (inner solve of a defect-correction
// step): the outer target atol + rtol*||r0|| is fixed by the first defect of
// the solve; an inner solve stops at the looser of that target and
// inner_rtol times its own initial norm, and a defect already below the
// target ends the outer loop.
__device__ __forceinline__ void start_eps(KScalars* S, double rNorm) {
    if (!S->mixed) {
        S->eps = S->atol + S->rtol * rNorm;
        return;
    }
    if (S->outer == 0) S->eps_outer = S->atol + S->rtol * rNorm;
    S->eps = fmax(S->eps_outer, S->inner_rtol * rNorm);
    S->outer_conv = rNorm <= S->eps_outer ? 1 : 0;
}

// CG direction buffers alternate: iteration k uses p_k = P[k & 1].  cg_start
// stores p_0 = z in P[0]; for k >= 1 the SpMV forms p_k = z + beta*p_{k-1}
// on the fly (Krylov.jl kaxpby!(n, 1, z, beta, p) -- the same expression for
// every reader, so gathered neighbours see bit-identical values) and the
// thread owning a row stores it.  The separate p-update pass disappears.
template <class T>
__device__ __forceinline__ T cg_dir(const T* __restrict__ z, const T* __restrict__ pold, T beta, int j) {
    return z[j] + beta * pold[j];
}

template <class T>
__device__ __forceinline__ void spmv_body(const TileCtx& tc, CSRView A, const T* __restrict__ nz,
                                                      const T* __restrict__ x, T* y, const KScalars* S) {
    if (S && S->done) return;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < A.n) y[i] = row_dot(A, nz, x, i);
    }
}

template <class T>
__device__ __forceinline__ void jacobi_apply_body(const TileCtx& tc, int n, const T* __restrict__ P, const T* __restrict__ r, T* z, const KScalars* S) {
    if (S && S->done) return;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < n) z[i] = P[i] * r[i];
    }
}

template <class T>
__device__ __forceinline__ void copy_body(const TileCtx& tc, int n, const T* __restrict__ a, T* b, const KScalars* S) {
    if (S && S->done) return;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < n) b[i] = a[i];
    }
}

// the start of a cg! solve from gamma = <r0, z0> (Krylov.jl cg!): norms,
// the stopping tolerance (start_eps), zero right-hand side, immediate stop
__device__ __forceinline__ void cg_start_scalars(KScalars* S, double gamma) {
    S->gamma = gamma;
    double rNorm = sqrt(gamma);
    S->rNorm = rNorm;
    S->rNorm0 = rNorm;
    S->iter = 0;
    S->done = 0;
    S->status = KS_RUNNING;
    S->outer_conv = 0;
    S->loops = 0;
    if (gamma == 0.0) {
        S->done = 1;
        S->status = KS_ZERO_RHS;
        S->outer_conv = 1;
        return;
    }
    S->pNorm2 = gamma;
    start_eps(S, rNorm);
    if (rNorm <= S->eps) {
        S->done = 1;
        S->status = KS_SOLVED;
    } else if (S->iter >= S->itmax) {
        S->done = 1;
        S->status = KS_TIRED;
    }
}

template <class T>
__device__ __forceinline__ void cg_start_body(const TileCtx& tc, int n, const T* __restrict__ r, const T* __restrict__ z, T* p, KScalars* S,
                           double* part) {
    __shared__ double sm[8];
    double acc = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < n) {
            T zi = z[i];
            p[i] = zi;
            acc = acc + (double)r[i] * (double)zi;
        }
    }
    double tot = block_tree(acc, sm);
    if (threadIdx.x == 0) part[tc.tile] = tot;
    if (!last_block(&S->counter, tc.ntiles)) return;
    double gamma = reduce_partials(part, tc.ntiles, sm);
    if (threadIdx.x == 0) cg_start_scalars(S, gamma);
}

template <class T>
__device__ __forceinline__ void cg_spmv_body(const TileCtx& tc, CSRView A, const T* __restrict__ nz,
                                                         const T* __restrict__ z, T* P0, T* P1, T* q, KScalars* S,
                                                         double* part) {
    if (S->done) return;
    __shared__ double sm[8];
    const int it = S->iter;
    const T beta = (T)S->beta;
    T* pk = (it & 1) ? P1 : P0;
    const T* pold = (it & 1) ? P0 : P1;
    double acc = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < A.n) {
            T qi = T(0), pi;
            const int rb = row_base(A, i), e1 = rb + SELL_C * A.len[i];
            if (it == 0) {
                for (int e = rb; e < e1; e += SELL_C) qi = qi + ld_stream(nz + e) * pk[ld_stream(A.colval + e)];
                pi = pk[i];
            } else {
                for (int e = rb; e < e1; e += SELL_C)
                    qi = qi + ld_stream(nz + e) * cg_dir(z, pold, beta, ld_stream(A.colval + e));
                pi = cg_dir(z, pold, beta, i);
                pk[i] = pi;
            }
            q[i] = qi;
            acc = acc + (double)pi * (double)qi;
        }
    }
    double tot = block_tree(acc, sm);
    if (threadIdx.x == 0) part[tc.tile] = tot;
    if (!last_block(&S->counter, tc.ntiles)) return;
    double pAp = reduce_partials(part, tc.ntiles, sm);
    if (threadIdx.x == 0) {
        const double epsT = sizeof(T) == 8 ? 2.220446049250313e-16 : 1.1920928955078125e-07;  // eps(T)
        double lim = epsT * S->pNorm2;
        if (pAp <= lim && fabs(pAp) <= lim) {
            S->done = 1;
            S->status = KS_ZERO_CURV;
            return;
        }
        S->alpha = S->gamma / pAp;
    }
}

template <class T>
__device__ __forceinline__ void cg_update_body(const TileCtx& tc, int n, T* x, const T* __restrict__ P0, const T* __restrict__ P1, T* r,
                            const T* __restrict__ q, T* z, const T* __restrict__ P, int jacobi_fused, KScalars* S,
                            double* part) {
    if (S->done) return;
    __shared__ double sm[8];
    const T* p = (S->iter & 1) ? P1 : P0;
    const T alpha = (T)S->alpha;
    double acc = 0.0;
    if constexpr (sizeof(T) == 4) {
        // FP32: 4-byte elements leave too few bytes in flight per thread when
        // each row waits for its loads; issue all rows' loads first (same
        // arithmetic, same order of the sums).  Measured 18.4 -> 14.4 us on
        // 2M rows.
        if (jacobi_fused) {
            T xv[RED_ITEMS], pv[RED_ITEMS], rv[RED_ITEMS], qv[RED_ITEMS], Pv[RED_ITEMS];
#pragma unroll
            for (int k = 0; k < RED_ITEMS; ++k) {
                int i = tile_row(tc, k);
                if (i < n) {
                    xv[k] = ld_stream(x + i);
                    pv[k] = p[i];
                    rv[k] = r[i];
                    qv[k] = ld_stream(q + i);
                    Pv[k] = ld_stream(P + i);
                }
            }
#pragma unroll
            for (int k = 0; k < RED_ITEMS; ++k) {
                int i = tile_row(tc, k);
                if (i < n) {
                    __stcs(x + i, xv[k] + alpha * pv[k]);
                    T ri = rv[k] + (-alpha) * qv[k];
                    r[i] = ri;
                    T zi = Pv[k] * ri;
                    z[i] = zi;
                    acc = acc + (double)ri * (double)zi;
                }
            }
            double tot = block_tree(acc, sm);
            if (threadIdx.x == 0) part[tc.tile] = tot;
            if (!last_block(&S->counter, tc.ntiles)) return;
            double g = reduce_partials(part, tc.ntiles, sm);
            if (threadIdx.x == 0) cg_finalize(S, g);
            return;
        }
    }
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < n) {
            // x, q and P are not read again before the next update: evict-first
            // keeps L2 for z and p, which the next SpMV gathers
            __stcs(x + i, ld_stream(x + i) + alpha * p[i]);
            T ri = r[i] + (-alpha) * ld_stream(q + i);
            r[i] = ri;
            if (jacobi_fused) {
                T zi = ld_stream(P + i) * ri;
                z[i] = zi;
                acc = acc + (double)ri * (double)zi;
            }
        }
    }
    if (!jacobi_fused) return;
    double tot = block_tree(acc, sm);
    if (threadIdx.x == 0) part[tc.tile] = tot;
    if (!last_block(&S->counter, tc.ntiles)) return;
    double g = reduce_partials(part, tc.ntiles, sm);
    if (threadIdx.x == 0) cg_finalize(S, g);
}

template <class T>
__device__ __forceinline__ void cg_rz_body(const TileCtx& tc, int n, const T* __restrict__ r, const T* __restrict__ z, KScalars* S, double* part) {
    if (S->done) return;
    __shared__ double sm[8];
    double acc = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < n) acc = acc + (double)r[i] * (double)z[i];
    }
    double tot = block_tree(acc, sm);
    if (threadIdx.x == 0) part[tc.tile] = tot;
    if (!last_block(&S->counter, tc.ntiles)) return;
    double g = reduce_partials(part, tc.ntiles, sm);
    if (threadIdx.x == 0) cg_finalize(S, g);
}

template <class T>
__device__ __forceinline__ void bicg_start_body(const TileCtx& tc, int n, const T* __restrict__ c, const T* __restrict__ r, T* p, KScalars* S,
                             double* part0, double* part1) {
    __shared__ double sm[8];
    double a0 = 0.0, a1 = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < n) {
            T ri = r[i];
            p[i] = ri;
            a0 = a0 + (double)ri * (double)ri;
            a1 = a1 + (double)c[i] * (double)ri;
        }
    }
    double t0 = block_tree(a0, sm);
    double t1 = block_tree(a1, sm);
    if (threadIdx.x == 0) {
        part0[tc.tile] = t0;
        part1[tc.tile] = t1;
    }
    if (!last_block(&S->counter, tc.ntiles)) return;
    double rr = reduce_partials(part0, tc.ntiles, sm);
    double cr = reduce_partials(part1, tc.ntiles, sm);
    if (threadIdx.x == 0) {
        double rNorm = sqrt(rr);
        S->rNorm = rNorm;
        S->rNorm0 = rNorm;
        S->iter = 0;
        S->done = 0;
        S->status = KS_RUNNING;
        S->outer_conv = 0;
        S->loops = 0;
        if (rNorm == 0.0) {
            S->done = 1;
            S->status = KS_ZERO_RHS;
            S->outer_conv = 1;
            return;
        }
        start_eps(S, rNorm);
        S->next_rho = cr;
        if (cr == 0.0) {
            S->done = 1;
            S->status = KS_BREAKDOWN;
            return;
        }
        if (rNorm <= S->eps) {
            S->done = 1;
            S->status = KS_SOLVED;
        } else if (S->iter >= S->itmax) {
            S->done = 1;
            S->status = KS_TIRED;
        }
    }
}

template <class T>
__device__ __forceinline__ void bicg_alpha_body(const TileCtx& tc, int n, const T* __restrict__ c, const T* __restrict__ v, KScalars* S, double* part) {
    if (S->done) return;
    __shared__ double sm[8];
    double acc = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < n) acc = acc + (double)c[i] * (double)v[i];
    }
    double tot = block_tree(acc, sm);
    if (threadIdx.x == 0) part[tc.tile] = tot;
    if (!last_block(&S->counter, tc.ntiles)) return;
    double cv = reduce_partials(part, tc.ntiles, sm);
    if (threadIdx.x == 0) {
        S->iter = S->iter + 1;
        S->rho = S->next_rho;
        S->cv = cv;
        S->alpha = S->rho / cv;
    }
}

template <class T>
__device__ __forceinline__ void bicg_s_body(const TileCtx& tc, int n, const T* __restrict__ r, const T* __restrict__ v, const T* __restrict__ p, T* s,
                         T* x, const KScalars* S) {
    if (S->done) return;
    const T alpha = (T)S->alpha;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < n) {
            s[i] = r[i] + (-alpha) * v[i];
            x[i] = x[i] + alpha * p[i];
        }
    }
}

template <class T>
__device__ __forceinline__ void bicg_omega_body(const TileCtx& tc, int n, const T* __restrict__ t, const T* __restrict__ s, KScalars* S, double* part0,
                             double* part1) {
    if (S->done) return;
    __shared__ double sm[8];
    double a0 = 0.0, a1 = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < n) {
            double ti = (double)t[i];
            a0 = a0 + ti * (double)s[i];
            a1 = a1 + ti * ti;
        }
    }
    double t0 = block_tree(a0, sm);
    double t1 = block_tree(a1, sm);
    if (threadIdx.x == 0) {
        part0[tc.tile] = t0;
        part1[tc.tile] = t1;
    }
    if (!last_block(&S->counter, tc.ntiles)) return;
    double ts = reduce_partials(part0, tc.ntiles, sm);
    double tt = reduce_partials(part1, tc.ntiles, sm);
    if (threadIdx.x == 0) S->omega = ts / tt;
}

template <class T>
__device__ __forceinline__ void bicg_xr_body(const TileCtx& tc, int n, T* x, const T* __restrict__ s, const T* __restrict__ t, T* r,
                          const T* __restrict__ c, KScalars* S, double* part0, double* part1) {
    if (S->done) return;
    __shared__ double sm[8];
    const double omega = S->omega;
    const T om = (T)omega;
    double a0 = 0.0, a1 = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < n) {
            T si = s[i];
            x[i] = x[i] + om * si;
            T ri = si + (-om) * t[i];
            r[i] = ri;
            a0 = a0 + (double)c[i] * (double)ri;
            a1 = a1 + (double)ri * (double)ri;
        }
    }
    double t0 = block_tree(a0, sm);
    double t1 = block_tree(a1, sm);
    if (threadIdx.x == 0) {
        part0[tc.tile] = t0;
        part1[tc.tile] = t1;
    }
    if (!last_block(&S->counter, tc.ntiles)) return;
    double cr = reduce_partials(part0, tc.ntiles, sm);
    double rr = reduce_partials(part1, tc.ntiles, sm);
    if (threadIdx.x == 0) {
        S->next_rho = cr;
        S->beta = (cr / S->rho) * (S->alpha / omega);
        double rNorm = sqrt(rr);
        S->rNorm = rNorm;
        bool mach = (rNorm + 1.0 <= 1.0);
        bool solved = (rNorm <= S->eps) || mach;
        bool tired = S->iter >= S->itmax;
        bool breakdown = (S->alpha == 0.0) || isnan(S->alpha);
        if (solved) {
            S->done = 1;
            S->status = KS_SOLVED;
        } else if (tired) {
            S->done = 1;
            S->status = KS_TIRED;
        } else if (breakdown) {
            S->done = 1;
            S->status = KS_BREAKDOWN;
        }
    }
}

template <class T>
__device__ __forceinline__ void bicg_p_body(const TileCtx& tc, int n, const T* __restrict__ r, const T* __restrict__ v, T* p, const KScalars* S) {
    if (S->done) return;
    const T beta = (T)S->beta, omega = (T)S->omega;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < n) p[i] = r[i] + beta * (p[i] + (-omega) * v[i]);
    }
}

// forward_substitution! row i (preconditioners_1_DILU.jl:84-98)
template <class T>
__device__ __forceinline__ void dilu_fwd_row(const CSRView& A, const T* __restrict__ nz, const T* __restrict__ D,
                                             const T* __restrict__ b, T* y, int i) {
    int ds = A.diag[i];
    T sum = T(0);
    for (int e = row_base(A, i); e < ds; e += SELL_C) {
        int j = ld_stream(A.colval + e);
        sum = sum + (ld_stream(nz + e) * y[j]) * (T(1) / D[j]);
    }
    y[i] = b[i] - sum;
}

// backward_substitution! row i (preconditioners_1_DILU.jl:100-114), in place
template <class T>
__device__ __forceinline__ void dilu_bwd_row(const CSRView& A, const T* __restrict__ nz, const T* __restrict__ D,
                                             T* x, int i) {
    int ds = A.diag[i];
    T sum = T(0);
    int e1 = row_base(A, i) + SELL_C * A.len[i];
    for (int e = ds + SELL_C; e < e1; e += SELL_C) sum = sum + ld_stream(nz + e) * x[ld_stream(A.colval + e)];
    x[i] = (x[i] - sum) / D[i];
}

// A DILU application of a small system (n <= DILU_BLOCK_MAX_ROWS) as one
// block: every level of the forward sweep, then of the backward sweep, with a
// block barrier between levels (rows of a level are independent).  It reads
// the level-ordered triangles (position k of level order: cnt[k] slots at
// slice[k/32] + k%32 + 32 j, coalesced across a warp) and, in the forward
// sweep, dinv = T(1)/D[col] per slot, so a row's loads do not wait on one
// another and no division sits on the sweep's critical path; ys is y
// itself or, when y fits, a shared-memory copy written back at the end.
// Per row the arithmetic is forward_substitution! / backward_substitution!
// (preconditioners_1_DILU.jl:84-114) in the row's own entry order:
//   forward  y_i = b_i - sum_j (a_ij y_j) (1/D_j)      (j < i)
//   backward x_i = (x_i - sum_j a_ij x_j) / D_i        (j > i)
// -- the values of the CSR-row sweeps (dilu_fwd_row / dilu_bwd_row), bit
// for bit.
constexpr int DILU_BLOCK_THREADS = 1024;

// One level of a sweep over level positions k0..k1.  FP32: each thread
// takes the rows k and k + blockDim.x together (all their slot loads issued
// before either row's sum), so a level wider than the block costs one
// dependent load chain per pair of rows, not per row; FP64 keeps one row at a
// time (two rows' registers spill at 1024 threads).  LOWER: forward
// substitution (y_i = b_i - sum (a_ij y_j) (1/D_j)); else backward (x_i =
// (x_i - sum a_ij x_j) / D_i).  The first U slots of a row sit in registers,
// the rest are read in a loop; each row's sum runs in its own entry order.
// (start, stride): the thread's first position and the stride between its
// positions -- the block (threadIdx.x, blockDim.x) for one-block sweeps, the
// grid for sweeps spread over every block (k_dilu_grid).
template <class T, bool LOWER>
__device__ __forceinline__ void dilu_level_s(const LevelView<T>& L, int k0, int k1, const T* __restrict__ D,
                                             const T* __restrict__ b, T* ys, int start, int stride) {
    constexpr int R = sizeof(T) == 4 ? 2 : 1;  // rows per thread per step
    constexpr int U = sizeof(T) == 4 ? 6 : 8;
    for (int k = k0 + start; k < k1; k += R * stride) {
        int kk[R];
#pragma unroll
        for (int r = 0; r < R; ++r) kk[r] = k + r * stride;
        int i[R], c[R], base[R];
        T rhs[R];
        int cj[R][U];
        T vj[R][U], dj[R][U];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            c[r] = 0;
            i[r] = 0;
            base[r] = 0;
            rhs[r] = T(0);
            if (kk[r] < k1) {
                i[r] = L.rows[kk[r]];
                c[r] = L.cnt[kk[r]];
                base[r] = L.slice[kk[r] / SELL_C] + (kk[r] % SELL_C);
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (kk[r] < k1) rhs[r] = LOWER ? b[i[r]] : D[i[r]];
#pragma unroll
            for (int j = 0; j < U; ++j)
                if (j < c[r]) {
                    const int e = base[r] + SELL_C * j;
                    cj[r][j] = ld_stream(L.col + e);
                    vj[r][j] = ld_stream(L.val + e);
                    if (LOWER) dj[r][j] = ld_stream(L.dinv + e);
                }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (kk[r] >= k1) continue;
            T sum = T(0);
#pragma unroll
            for (int j = 0; j < U; ++j)
                if (j < c[r]) sum = LOWER ? sum + (vj[r][j] * ys[cj[r][j]]) * dj[r][j] : sum + vj[r][j] * ys[cj[r][j]];
            for (int j = U; j < c[r]; ++j) {
                const int e = base[r] + SELL_C * j;
                sum = LOWER ? sum + (ld_stream(L.val + e) * ys[ld_stream(L.col + e)]) * ld_stream(L.dinv + e)
                            : sum + ld_stream(L.val + e) * ys[ld_stream(L.col + e)];
            }
            ys[i[r]] = LOWER ? rhs[r] - sum : (ys[i[r]] - sum) / rhs[r];
        }
    }
}

template <class T, bool LOWER>
__device__ __forceinline__ void dilu_level(const LevelView<T>& L, int k0, int k1, const T* __restrict__ D,
                                           const T* __restrict__ b, T* ys) {
    dilu_level_s<T, LOWER>(L, k0, k1, D, b, ys, (int)threadIdx.x, (int)blockDim.x);
}

template <class T>
__device__ __forceinline__ void dilu_level_sweep(int n, const LevelView<T>& lo, const LevelView<T>& up,
                                                 const T* __restrict__ D, const T* __restrict__ b, T* y, T* ys) {
    for (int l = 0; l < lo.nlev; ++l) {
        dilu_level<T, true>(lo, lo.off[l], lo.off[l + 1], D, b, ys);
        __syncthreads();
    }
    for (int l = 0; l < up.nlev; ++l) {
        dilu_level<T, false>(up, up.off[l], up.off[l + 1], D, b, ys);
        __syncthreads();
    }
    if (ys != y)
        for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = ys[i];
}

// update_dilu_diagonal! row i (preconditioners_1_DILU.jl:43-82)
__device__ __forceinline__ void dilu_D_row(const CSRView& A, const double* __restrict__ nz, double* D, int i) {
    int ds = A.diag[i];
    double d = nz[ds];
    for (int e = row_base(A, i); e < ds; e += SELL_C) {
        int j = A.colval[e];
        d = d - (nz[A.trans[e]] * nz[e]) / D[j];
    }
    D[i] = d;
}

// ---- persistent CG (Jacobi or no preconditioner) ----
// Grid-wide barrier among the nblocks co-resident blocks of one system.
// `count` only grows during a launch (zeroed before it): barrier number nb
// completes when it reaches (nb + 1) * nblocks, so there is no reset and no
// second atomic.  Thread 0 alone arrives, with a release reduction (the
// block's writes, ordered before it by __syncthreads, become visible with
// it), and polls with acquire loads; __syncthreads orders the rest of the
// block after it.  (Measured alone on B200: 1.6 us per barrier among 148
// blocks, against 2.0 us with full fences around a relaxed atomic.)  A
// single-block system needs no more than the __syncthreads.  Bounded: a
// block that polls more than BAR_SPIN_LIMIT times, or sees *err set by
// another block, returns false (and sets *err), so a failure ends every
// block within one bounded wait.
constexpr long BAR_SPIN_LIMIT = 1L << 22;
__device__ __forceinline__ void red_release_add(unsigned int* p, unsigned int v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ bool grid_barrier(unsigned int* count, int nblocks, unsigned int& nb, int* err,
                                             int* sh_err, long spin_limit = BAR_SPIN_LIMIT) {
    __syncthreads();
    if (nblocks == 1) return true;
    if (threadIdx.x == 0) {
        const unsigned int target = (nb + 1u) * (unsigned int)nblocks;
        red_release_add(count, 1u);
        long spins = 0;
        int e = 0;
        while ((int)(ld_acquire(count) - target) < 0) {
            if (++spins > spin_limit) {
                e = 1;
                *(volatile int*)err = 1;
                break;
            }
            if ((spins & 255) == 0 && *(volatile int*)err) {
                e = 1;
                break;
            }
            __nanosleep(32);
        }
        *sh_err = e;
    }
    ++nb;
    __syncthreads();
    return *sh_err == 0;
}

// q_i = sum_k nz[i,k] * d[col(i,k)] in slot order, d = p (first iteration) or
// z + beta p_old gathered on the fly: the first 8 slots' loads are issued
// together, the products are then added in slot order (wide form only; the
// narrow form keeps the plain loop, which needs fewer registers).
template <class T, bool FIRST>
__device__ __forceinline__ T cg_row_q(const CSRView& A, const T* __restrict__ nz, const T* z, const T* pold,
                                      const T* pk, T b, int i) {
    const int rb = row_base(A, i), ln = A.len[i];
    T qi = T(0);
    int c[8];
    T v[8];
#pragma unroll
    for (int t = 0; t < 8; ++t)
        if (t < ln) {
            c[t] = ld_stream(A.colval + rb + SELL_C * t);
            v[t] = ld_stream(nz + rb + SELL_C * t);
        }
#pragma unroll
    for (int t = 0; t < 8; ++t)
        if (t < ln) qi = qi + v[t] * (FIRST ? pk[c[t]] : cg_dir(z, pold, b, c[t]));
    for (int t = 8; t < ln; ++t) {
        const int s = rb + SELL_C * t;
        const int cc = ld_stream(A.colval + s);
        qi = qi + ld_stream(nz + s) * (FIRST ? pk[cc] : cg_dir(z, pold, b, cc));
    }
    return qi;
}

// Bulk prefetch of [p, p + bytes) into L2 (no data reaches the SM; p and
// bytes 16-byte multiples)
__device__ __forceinline__ void l2_prefetch(const void* p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// __launch_bounds__ minimum blocks per SM of each form: 64 registers for the
// wide forms, 32 for the narrow one (8 blocks of 256 threads per SM)
constexpr int persist_min_blocks(int nt) { return nt == 1024 ? 1 : nt == 512 ? 2 : 8; }

// The whole CG loop of Krylov.jl cg! (Jacobi-fused update) for one system,
// run by its ntiles blocks (block with tile t owns canonical tile t); per
// iteration
//   phase 1: p_k = z + beta p_{k-1} (gathered), q = A p_k for the tile's rows,
//            q kept in shared memory, p_k stored; tile partial of <p_k, q>;
//   barrier; every block reduces the partials (same tree) -> alpha, zero-
//            curvature test (identical decisions in every block);
//   phase 2: x += alpha p_k, r -= alpha q, z = P r; tile partial of <r, z>;
//   barrier; every block reduces -> cg! stopping tests, beta.
// The arithmetic is that of k_cg_spmv + k_cg_update; q never goes to HBM and
// the two kernel boundaries per iteration disappear.  The block of tile 0
// writes the scalar state back.  Runs at most max_iters iterations.  The
// barriers count only this system's blocks, so in a batched launch every
// system runs (and finishes) on its own.
//
// NT threads per block.  NT = RED_THREADS (narrow): thread t owns the tile's
// rows t + 256 k, k < 8, and accumulates its partial as it goes -- few
// registers, so 7-8 blocks fit an SM and a 2M-row system is co-resident.
// NT = 512 / 1024 (wide, for systems of at most 2 / 1 tiles per SM): thread
// t covers rows (t mod 256) + 256 k for NT/256 times fewer k, writes each
// row's product to shared memory, and threads 0..255 then add the products
// of "their" rows in k order -- the same partials, bit for bit, with a 4-8x
// shorter dependent-load chain per thread.
//
// Narrow form only: while a block waits at a barrier, the data its next
// phase streams is already being pulled into L2 -- x, r and P of its rows
// before the first barrier, and (pf_kb > 0, for matrices that fit L2) up to
// pf_kb KB of its matrix slots before the second.  Measured on B200 at 96^3
// / 128^3 (FP64): the vectors 5% / 1.7% faster; the matrix another 5% at
// 96^3 but 15% slower at 128^3 (it evicts the gathered vectors), hence the
// size condition.
// The canonical final tree over the tile partials of a system whose blocks
// form one thread-block cluster: thread t < T reads block t's partial from
// its shared memory (the values reduce_partials reads from global memory).
__device__ __forceinline__ double reduce_cluster(double* mine, int T, double* smem8) {
    double s = 0.0;
    if (threadIdx.x < RED_THREADS)
        for (int i = threadIdx.x; i < T; i += RED_THREADS)
            s = s + *cooperative_groups::this_cluster().map_shared_rank(mine, i);
    return block_tree(s, smem8);
}

// CL (cluster form, wide blocks only): the system's tiles are the blocks of
// one thread-block cluster (blocks past its tile count have no rows); the
// barriers are hardware cluster barriers (release / acquire at cluster
// scope) and the partials travel through distributed shared memory -- no
// global spin, no atomics, no cooperative launch (clusters are scheduled
// whole), and each cluster runs on its own.  Every block takes the same
// decisions, so all reach the same barriers; a last barrier keeps every
// block's shared memory alive until its peers have read it.
template <class T, int NT, bool CL = false>
__device__ __forceinline__ void cg_persist_body(const TileCtx& tc, const CSRView& A, const T* __restrict__ nz,
                                                const T* __restrict__ Pj, int jacobi, T* x, T* r, T* z, T* P0,
                                                T* P1, KScalars* S, double* part, double* part2, unsigned int* bar,
                                                int* err, int max_iters, int pf_kb) {
    constexpr bool WIDE = NT > RED_THREADS;
    static_assert(!CL || WIDE, "the cluster form uses wide blocks");
    __shared__ double cl_part[2];  // cluster form: this block's two tile partials
    constexpr int IPT = RED_ITEMS / (NT / RED_THREADS);  // rows per thread
    __shared__ T q_s[RED_TILE];
    __shared__ double pr_s[WIDE ? RED_TILE : 1];
    __shared__ double sm[8];
    __shared__ double sh_d[4];
    __shared__ int sh_i[3];
    __shared__ int sh_err;
    const int n = A.n;
    const int v = threadIdx.x & (RED_THREADS - 1), k0 = (threadIdx.x / RED_THREADS) * IPT;
    int iter = S->iter, done = S->done, status = S->status;
    const int itmax = S->itmax;
    double gamma = S->gamma, beta = S->beta, pNorm2 = S->pNorm2, alpha = S->alpha, rNorm = S->rNorm;
    const double eps = S->eps;
    const double epsT = sizeof(T) == 8 ? 2.220446049250313e-16 : 1.1920928955078125e-07;  // eps(T)
    int ran = 0;
    unsigned int nb = 0;
    bool ok = true;
    while (!done && ran < max_iters) {
        // phase 1: q = A p_k (k_cg_spmv)
        T* pk = (iter & 1) ? P1 : P0;
        const T* pold = (iter & 1) ? P0 : P1;
        const T b = (T)beta;
        double acc = 0.0;
        if constexpr (!WIDE) {
            for (int k = 0; k < RED_ITEMS; ++k) {
                int i = tile_row(tc, k);
                if (i < n) {
                    T qi = T(0), pi;
                    const int rb = row_base(A, i), e1 = rb + SELL_C * A.len[i];
                    if (iter == 0) {
                        for (int e = rb; e < e1; e += SELL_C)
                            qi = qi + ld_stream(nz + e) * pk[ld_stream(A.colval + e)];
                        pi = pk[i];
                    } else {
                        for (int e = rb; e < e1; e += SELL_C)
                            qi = qi + ld_stream(nz + e) * cg_dir(z, pold, b, ld_stream(A.colval + e));
                        pi = cg_dir(z, pold, b, i);
                        pk[i] = pi;
                    }
                    q_s[k * RED_THREADS + threadIdx.x] = qi;
                    acc = acc + (double)pi * (double)qi;
                }
            }
        } else {
            // rows past n contribute 0.0 to the k-ordered sums below: the
            // narrow form skips them, and x + 0.0 == x for every partial
            // sum that starts at +0.0 (it can never be -0.0)
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const int k = k0 + j, i = tc.tile * RED_TILE + k * RED_THREADS + v;
                double prod = 0.0;
                if (i < n) {
                    T qi, pi;
                    if (iter == 0) {
                        qi = cg_row_q<T, true>(A, nz, z, pold, pk, b, i);
                        pi = pk[i];
                    } else {
                        qi = cg_row_q<T, false>(A, nz, z, pold, pk, b, i);
                        pi = cg_dir(z, pold, b, i);
                        pk[i] = pi;
                    }
                    q_s[k * RED_THREADS + v] = qi;
                    prod = (double)pi * (double)qi;
                }
                pr_s[k * RED_THREADS + v] = prod;
            }
            __syncthreads();
            if (threadIdx.x < RED_THREADS)
#pragma unroll
                for (int k = 0; k < RED_ITEMS; ++k) acc = acc + pr_s[k * RED_THREADS + v];
        }
        double tot = block_tree(acc, sm);
        if (threadIdx.x == 0) {
            if constexpr (CL)
                cl_part[0] = tot;
            else
                part[tc.tile] = tot;
        }
        if (!WIDE && threadIdx.x < 3 && (threadIdx.x < 2 || jacobi)) {
            const long r0 = (long)tc.tile * RED_TILE;
            const long nr = min((long)RED_TILE, (long)n - r0);
            const unsigned bytes = (unsigned)((nr * (long)sizeof(T)) & ~15L);
            const T* base = threadIdx.x == 0 ? x : threadIdx.x == 1 ? r : Pj;
            if (bytes) l2_prefetch(base + r0, bytes);
        }
        if constexpr (CL)
            cooperative_groups::this_cluster().sync();
        else if (!(ok = grid_barrier(bar, tc.ntiles, nb, err, &sh_err)))
            break;
        double pAp = CL ? reduce_cluster(&cl_part[0], tc.ntiles, sm) : reduce_partials(part, tc.ntiles, sm);
        if (threadIdx.x == 0) {
            double lim = epsT * pNorm2;
            sh_i[0] = (pAp <= lim && fabs(pAp) <= lim) ? 1 : 0;
            sh_d[0] = gamma / pAp;
        }
        __syncthreads();
        if (sh_i[0]) {
            done = 1;
            status = KS_ZERO_CURV;
            break;
        }
        alpha = sh_d[0];
        // phase 2: x, r, z and <r, z> (k_cg_update, Jacobi fused)
        const T a = (T)alpha;
        double acc2 = 0.0;
        if constexpr (!WIDE) {
            for (int k = 0; k < RED_ITEMS; ++k) {
                int i = tile_row(tc, k);
                if (i < n) {
                    __stcs(x + i, ld_stream(x + i) + a * pk[i]);
                    T ri = r[i] + (-a) * q_s[k * RED_THREADS + threadIdx.x];
                    r[i] = ri;
                    T zi = jacobi ? ld_stream(Pj + i) * ri : ri;
                    if (jacobi) z[i] = zi;
                    acc2 = acc2 + (double)ri * (double)zi;
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const int k = k0 + j, i = tc.tile * RED_TILE + k * RED_THREADS + v;
                double prod = 0.0;
                if (i < n) {
                    __stcs(x + i, ld_stream(x + i) + a * pk[i]);
                    T ri = r[i] + (-a) * q_s[k * RED_THREADS + v];
                    r[i] = ri;
                    T zi = jacobi ? ld_stream(Pj + i) * ri : ri;
                    if (jacobi) z[i] = zi;
                    prod = (double)ri * (double)zi;
                }
                pr_s[k * RED_THREADS + v] = prod;
            }
            __syncthreads();
            if (threadIdx.x < RED_THREADS)
#pragma unroll
                for (int k = 0; k < RED_ITEMS; ++k) acc2 = acc2 + pr_s[k * RED_THREADS + v];
        }
        double tot2 = block_tree(acc2, sm);
        if (threadIdx.x == 0) {
            if constexpr (CL)
                cl_part[1] = tot2;
            else
                part2[tc.tile] = tot2;
        }
        if (!WIDE && pf_kb > 0 && threadIdx.x < 32) {
            // the tile's slots are contiguous: slices s0 .. s1 (16 KB pieces;
            // lanes 0..15 the values, 16..31 the columns)
            const int s0 = tc.tile * (RED_TILE / SELL_C);
            const int s1 = min(s0 + RED_TILE / SELL_C, (n + SELL_C - 1) / SELL_C);
            const long e0 = A.slice[s0], e1 = A.slice[s1];
            const bool vals = threadIdx.x < 16;
            const char* p0 = vals ? (const char*)(nz + e0) : (const char*)(A.colval + e0);
            const long span = (e1 - e0) * (vals ? (long)sizeof(T) : 4L);
            const long lim = min(span, (long)pf_kb * (vals ? 1024L : 512L));
            for (long o = (threadIdx.x & 15) * 16384L; o < lim; o += 16 * 16384L) {
                const unsigned bytes = (unsigned)(min(16384L, lim - o) & ~15L);
                if (bytes) l2_prefetch(p0 + o, bytes);
            }
        }
        if constexpr (CL)
            cooperative_groups::this_cluster().sync();
        else if (!(ok = grid_barrier(bar, tc.ntiles, nb, err, &sh_err)))
            break;
        double g = CL ? reduce_cluster(&cl_part[1], tc.ntiles, sm) : reduce_partials(part2, tc.ntiles, sm);
        if (threadIdx.x == 0) {  // cg_finalize on the block's copy of the state
            double rn = sqrt(g);
            bool mach = (rn + 1.0 <= 1.0);
            bool solved = (rn <= eps) || mach;
            double bt = beta, pn = pNorm2, gm = gamma;
            if (!solved) {
                bt = g / gamma;
                pn = g + (bt * bt) * pNorm2;
                gm = g;
            }
            int it1 = iter + 1;
            int dn = 0, stt = status;
            if (solved) {
                dn = 1;
                stt = KS_SOLVED;
            } else if (it1 >= itmax) {
                dn = 1;
                stt = KS_TIRED;
            }
            sh_d[0] = rn;
            sh_d[1] = bt;
            sh_d[2] = pn;
            sh_d[3] = gm;
            sh_i[0] = it1;
            sh_i[1] = dn;
            sh_i[2] = stt;
        }
        __syncthreads();
        rNorm = sh_d[0];
        beta = sh_d[1];
        pNorm2 = sh_d[2];
        gamma = sh_d[3];
        iter = sh_i[0];
        done = sh_i[1];
        status = sh_i[2];
        ++ran;
    }
    if constexpr (CL) cooperative_groups::this_cluster().sync();
    if (ok && tc.tile == 0 && threadIdx.x == 0) {
        S->iter = iter;
        S->done = done;
        S->status = status;
        S->gamma = gamma;
        S->beta = beta;
        S->pNorm2 = pNorm2;
        S->alpha = alpha;
        S->rNorm = rNorm;
    }
}

// The same CG loop with one block per SM, each block owning the canonical
// tiles t = blockIdx.x, blockIdx.x + G, ... (G blocks): per tile and phase it
// runs the wide form's rows (NT / 256 row groups per tile, the rows'
// products in k order by threads 0..255) and writes the tile's partial, so
// the partials -- and every value -- are those of one block per tile, bit
// for bit.  Only G blocks meet at each grid barrier (148 instead of one per
// 2048-row tile), and each thread issues a row's slot loads together.  q of
// all the block's tiles stays in shared memory (dynamic, tpb tiles).
template <class T, int NT>
__device__ __forceinline__ void cg_persist_mt_body(const CSRView& A, const T* __restrict__ nz,
                                                   const T* __restrict__ Pj, int jacobi, T* x, T* r, T* z, T* P0,
                                                   T* P1, KScalars* S, double* part, double* part2,
                                                   unsigned int* bar, int* err, int max_iters, T* q_s) {
    static_assert(NT > RED_THREADS, "one block covers a tile's rows in NT / 256 groups");
    constexpr int IPT = RED_ITEMS / (NT / RED_THREADS);  // rows per thread and tile
    __shared__ double pr_s[RED_TILE];
    __shared__ double sm[8];
    __shared__ double sh_d[4];
    __shared__ int sh_i[3];
    __shared__ int sh_err;
    const int n = A.n;
    const int ntiles = (n + RED_TILE - 1) / RED_TILE;
    const int G = gridDim.x;
    const int v = threadIdx.x & (RED_THREADS - 1), k0 = (threadIdx.x / RED_THREADS) * IPT;
    int iter = S->iter, done = S->done, status = S->status;
    const int itmax = S->itmax;
    double gamma = S->gamma, beta = S->beta, pNorm2 = S->pNorm2, alpha = S->alpha, rNorm = S->rNorm;
    const double eps = S->eps;
    const double epsT = sizeof(T) == 8 ? 2.220446049250313e-16 : 1.1920928955078125e-07;  // eps(T)
    int ran = 0;
    unsigned int nb = 0;
    bool ok = true;
    while (!done && ran < max_iters) {
        T* pk = (iter & 1) ? P1 : P0;
        const T* pold = (iter & 1) ? P0 : P1;
        const T b = (T)beta;
        // phase 1, tile by tile: q = A p_k into q_s, the tile's <p_k, q>
        for (int t = blockIdx.x, j = 0; t < ntiles; t += G, ++j) {
#pragma unroll
            for (int u = 0; u < IPT; ++u) {
                const int k = k0 + u, i = t * RED_TILE + k * RED_THREADS + v;
                double prod = 0.0;
                if (i < n) {
                    T qi, pi;
                    if (iter == 0) {
                        qi = cg_row_q<T, true>(A, nz, z, pold, pk, b, i);
                        pi = pk[i];
                    } else {
                        qi = cg_row_q<T, false>(A, nz, z, pold, pk, b, i);
                        pi = cg_dir(z, pold, b, i);
                        pk[i] = pi;
                    }
                    q_s[j * RED_TILE + k * RED_THREADS + v] = qi;
                    prod = (double)pi * (double)qi;
                }
                pr_s[k * RED_THREADS + v] = prod;
            }
            __syncthreads();
            double acc = 0.0;
            if (threadIdx.x < RED_THREADS)
#pragma unroll
                for (int k = 0; k < RED_ITEMS; ++k) acc = acc + pr_s[k * RED_THREADS + v];
            const double tot = block_tree(acc, sm);  // its barriers also free pr_s for the next tile
            if (threadIdx.x == 0) part[t] = tot;
        }
        if (!(ok = grid_barrier(bar, G, nb, err, &sh_err))) break;
        const double pAp = reduce_partials(part, ntiles, sm);
        if (threadIdx.x == 0) {
            const double lim = epsT * pNorm2;
            sh_i[0] = (pAp <= lim && fabs(pAp) <= lim) ? 1 : 0;
            sh_d[0] = gamma / pAp;
        }
        __syncthreads();
        if (sh_i[0]) {
            done = 1;
            status = KS_ZERO_CURV;
            break;
        }
        alpha = sh_d[0];
        // phase 2, tile by tile: x, r, z and the tile's <r, z>
        const T a = (T)alpha;
        for (int t = blockIdx.x, j = 0; t < ntiles; t += G, ++j) {
#pragma unroll
            for (int u = 0; u < IPT; ++u) {
                const int k = k0 + u, i = t * RED_TILE + k * RED_THREADS + v;
                double prod = 0.0;
                if (i < n) {
                    __stcs(x + i, ld_stream(x + i) + a * pk[i]);
                    T ri = r[i] + (-a) * q_s[j * RED_TILE + k * RED_THREADS + v];
                    r[i] = ri;
                    T zi = jacobi ? ld_stream(Pj + i) * ri : ri;
                    if (jacobi) z[i] = zi;
                    prod = (double)ri * (double)zi;
                }
                pr_s[k * RED_THREADS + v] = prod;
            }
            __syncthreads();
            double acc2 = 0.0;
            if (threadIdx.x < RED_THREADS)
#pragma unroll
                for (int k = 0; k < RED_ITEMS; ++k) acc2 = acc2 + pr_s[k * RED_THREADS + v];
            const double tot2 = block_tree(acc2, sm);
            if (threadIdx.x == 0) part2[t] = tot2;
        }
        if (!(ok = grid_barrier(bar, G, nb, err, &sh_err))) break;
        const double g = reduce_partials(part2, ntiles, sm);
        if (threadIdx.x == 0) {  // cg_finalize on the block's copy of the state
            const double rn = sqrt(g);
            const bool solved = (rn <= eps) || (rn + 1.0 <= 1.0);
            double bt = beta, pn = pNorm2, gm = gamma;
            if (!solved) {
                bt = g / gamma;
                pn = g + (bt * bt) * pNorm2;
                gm = g;
            }
            const int it1 = iter + 1;
            int dn = 0, stt = status;
            if (solved) {
                dn = 1;
                stt = KS_SOLVED;
            } else if (it1 >= itmax) {
                dn = 1;
                stt = KS_TIRED;
            }
            sh_d[0] = rn;
            sh_d[1] = bt;
            sh_d[2] = pn;
            sh_d[3] = gm;
            sh_i[0] = it1;
            sh_i[1] = dn;
            sh_i[2] = stt;
        }
        __syncthreads();
        rNorm = sh_d[0];
        beta = sh_d[1];
        pNorm2 = sh_d[2];
        gamma = sh_d[3];
        iter = sh_i[0];
        done = sh_i[1];
        status = sh_i[2];
        ++ran;
    }
    if (ok && blockIdx.x == 0 && threadIdx.x == 0) {
        S->iter = iter;
        S->done = done;
        S->status = status;
        S->gamma = gamma;
        S->beta = beta;
        S->pNorm2 = pNorm2;
        S->alpha = alpha;
        S->rNorm = rNorm;
    }
}

}  // namespace xcal
