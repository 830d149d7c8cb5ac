// krylov_bodies.cuh -- per-tile bodies of the Krylov kernels.
//
// Each body works on one canonical tile `tc.tile` of a system with
// `tc.ntiles` tiles.  The single-system kernels (kernels_krylov.cu) pass the
// grid (tile = block, ntiles = grid size); the batched kernels
// (kernels_batch.cu) pass a (system, local tile) entry of their tile map, so a
// system's arithmetic -- row sums, reduction trees, scalar decisions -- is the
// same whether it is solved alone or inside a batch.
#pragma once
#include "dev_common.cuh"

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
    if (threadIdx.x == 0) {
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
// block barrier between levels (rows of a level are independent).  The
// per-row arithmetic is the level kernels'.
constexpr int DILU_BLOCK_THREADS = 1024;

template <class T>
__device__ __forceinline__ void dilu_block_sweep(const CSRView& A, const T* __restrict__ nz, const T* __restrict__ D,
                                                 const T* __restrict__ in, T* out, const int* __restrict__ lo_rows,
                                                 const int* __restrict__ lo_off, int n_lo,
                                                 const int* __restrict__ up_rows, const int* __restrict__ up_off,
                                                 int n_up) {
    for (int l = 0; l < n_lo; ++l) {
        for (int k = lo_off[l] + threadIdx.x; k < lo_off[l + 1]; k += blockDim.x)
            dilu_fwd_row(A, nz, D, in, out, lo_rows[k]);
        __syncthreads();
    }
    for (int l = 0; l < n_up; ++l) {
        for (int k = up_off[l] + threadIdx.x; k < up_off[l + 1]; k += blockDim.x)
            dilu_bwd_row(A, nz, D, out, up_rows[k]);
        __syncthreads();
    }
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

}  // namespace xcal
