// kernels_krylov.cu -- Krylov solves of the hot path (FP64).
//
// CG and BiCGSTAB follow Krylov.jl 0.10 (cg!, bicgstab!; called from
// src/Solve/Solve_1_api.jl:286-289 with warm start, M = preconditioner,
// ldiv = true for DILU).  All scalars live on the device; each reduction is a
// canonical tile tree finished by the last block of the kernel, which also
// takes the algorithm's scalar decisions (step sizes, stopping tests), so the
// host only polls a `done` flag between chunks of iterations.
#include "dev_common.cuh"
#include "kernels.hpp"

namespace xcal {

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double row_dot(const CSRView& A, const double* __restrict__ nz,
                                          const double* __restrict__ x, int i) {
    // xmul! row (src/Multithread/spmvm.jl:47-53): sequential from 0.0
    double acc = 0.0;
    const int rb = row_base(A, i), rl = A.len[i];
    for (int k = 0; k < rl; ++k) {
        int e = rb + SELL_C * k;
        acc = acc + ld_stream(nz + e) * x[ld_stream(A.colval + e)];
    }
    return acc;
}

// Tile SpMV: the thread owning canonical row k (row = tile*RED_TILE +
// k*RED_THREADS + t) sums that row sequentially in CSR order (the reference's
// row order).  Each thread only reads back its own rows, so the staging array
// needs no barrier.  (Measured on the 128^3 7-point pattern: one thread per
// row beats lane-grouped rows and smem-staged segments; with random numbering
// the x gathers, not the matrix stream, bound it.)
struct SpmvSmem {
    double q[RED_TILE];
};

__device__ __forceinline__ void tile_spmv(const CSRView& A, const double* __restrict__ nz,
                                          const double* __restrict__ x, SpmvSmem& sm) {
    const int row0 = blockIdx.x * RED_TILE;
    const int nrows = min(RED_TILE, A.n - row0);
#pragma unroll
    for (int k = 0; k < RED_ITEMS; ++k) {
        int r = k * RED_THREADS + threadIdx.x;
        if (r < nrows) sm.q[r] = row_dot(A, nz, x, row0 + r);
    }
}
// (A x) of the thread's canonical row k (valid after tile_spmv)
__device__ __forceinline__ double tile_q(const SpmvSmem& sm, int k) { return sm.q[k * RED_THREADS + threadIdx.x]; }

// CG stopping decisions after gamma_next = <r,z> (Krylov.jl cg!)
__device__ void cg_finalize(KScalars* S, double gamma_next) {
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

// ---------------------------------------------------------------------------
// kernels (grid = one canonical tile per block, RED_THREADS threads)
// ---------------------------------------------------------------------------
// r = b - A*x0, x = 0, dx = x0 (warm start: Krylov.jl kaxpby!(n,1,b,-1,r))
__global__ void __launch_bounds__(RED_THREADS, 8) k_init_resid(CSRView A, const double* __restrict__ nz,
                                                            const double* __restrict__ b,
                                                            const double* __restrict__ field, double* dx, double* x,
                                                            double* r) {
    __shared__ SpmvSmem sm;
    tile_spmv(A, nz, field, sm);
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < A.n) {
            r[i] = b[i] - tile_q(sm, k);
            x[i] = 0.0;
            dx[i] = field[i];
        }
    }
}

// y = A*x (plain SpMV, early exit when the solve is done)
__global__ void __launch_bounds__(RED_THREADS, 8) k_spmv(CSRView A, const double* __restrict__ nz,
                                                      const double* __restrict__ x, double* y, const KScalars* S) {
    if (S && S->done) return;
    __shared__ SpmvSmem sm;
    tile_spmv(A, nz, x, sm);
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < A.n) y[i] = tile_q(sm, k);
    }
}

// z = P .* r (Jacobi: opDiagonal multiply, ldiv = false)
__global__ void k_jacobi_apply(int n, const double* __restrict__ P, const double* __restrict__ r, double* z,
                               const KScalars* S) {
    if (S && S->done) return;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) z[i] = P[i] * r[i];
    }
}

__global__ void k_copy(int n, const double* __restrict__ a, double* b, const KScalars* S) {
    if (S && S->done) return;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) b[i] = a[i];
    }
}

// ---- CG ----
// p = z; gamma = <r,z>; initial stopping tests
__global__ void k_cg_start(int n, const double* __restrict__ r, const double* __restrict__ z, double* p,
                           KScalars* S, double* part) {
    __shared__ double sm[8];
    double acc = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) {
            double zi = z[i];
            p[i] = zi;
            acc = acc + r[i] * zi;
        }
    }
    double tot = block_tree(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
    if (!last_block(&S->counter)) return;
    double gamma = reduce_partials(part, gridDim.x, sm);
    if (threadIdx.x == 0) {
        S->gamma = gamma;
        double rNorm = sqrt(gamma);
        S->rNorm = rNorm;
        S->iter = 0;
        S->done = 0;
        S->status = KS_RUNNING;
        if (gamma == 0.0) {
            S->done = 1;
            S->status = KS_ZERO_RHS;
            return;
        }
        S->pNorm2 = gamma;
        S->eps = S->atol + S->rtol * rNorm;
        if (rNorm <= S->eps) {
            S->done = 1;
            S->status = KS_SOLVED;
        } else if (S->iter >= S->itmax) {
            S->done = 1;
            S->status = KS_TIRED;
        }
    }
}

// CG direction buffers alternate: iteration k uses p_k = P[k & 1].  cg_start
// stores p_0 = z in P[0]; for k >= 1 the SpMV forms p_k = z + beta*p_{k-1}
// on the fly (Krylov.jl kaxpby!(n, 1, z, beta, p) -- the same expression for
// every reader, so gathered neighbours see bit-identical values) and the
// thread owning a row stores it.  The separate p-update pass disappears.
__device__ __forceinline__ double cg_dir(const double* __restrict__ z, const double* __restrict__ pold, double beta,
                                         int j) {
    return z[j] + beta * pold[j];
}

// q = A p_k; pAp = <p_k,q>; zero-curvature test; alpha = gamma / pAp
__global__ void __launch_bounds__(RED_THREADS, 8) k_cg_spmv(CSRView A, const double* __restrict__ nz,
                                                         const double* __restrict__ z, double* P0, double* P1,
                                                         double* q, KScalars* S, double* part) {
    if (S->done) return;
    __shared__ double sm[8];
    const int it = S->iter;
    const double beta = S->beta;
    double* pk = (it & 1) ? P1 : P0;
    const double* pold = (it & 1) ? P0 : P1;
    double acc = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < A.n) {
            double qi = 0.0, pi;
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
            acc = acc + pi * qi;
        }
    }
    double tot = block_tree(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
    if (!last_block(&S->counter)) return;
    double pAp = reduce_partials(part, gridDim.x, sm);
    if (threadIdx.x == 0) {
        const double epsT = 2.220446049250313e-16;  // eps(Float64)
        double lim = epsT * S->pNorm2;
        if (pAp <= lim && fabs(pAp) <= lim) {
            S->done = 1;
            S->status = KS_ZERO_CURV;
            return;
        }
        S->alpha = S->gamma / pAp;
    }
}

// x += alpha p_k; r -= alpha q; [Jacobi: z = P r; <r,z>; finalize]
__global__ void k_cg_update(int n, double* x, const double* __restrict__ P0, const double* __restrict__ P1,
                            double* r, const double* __restrict__ q, double* z, const double* __restrict__ P,
                            int jacobi_fused, KScalars* S, double* part) {
    if (S->done) return;
    __shared__ double sm[8];
    const double* p = (S->iter & 1) ? P1 : P0;
    double alpha = S->alpha;
    double acc = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) {
            // x, q and P are not read again before the next update: evict-first
            // keeps L2 for z and p, which the next SpMV gathers
            __stcs(x + i, ld_stream(x + i) + alpha * p[i]);
            double ri = r[i] + (-alpha) * ld_stream(q + i);
            r[i] = ri;
            if (jacobi_fused) {
                double zi = ld_stream(P + i) * ri;
                z[i] = zi;
                acc = acc + ri * zi;
            }
        }
    }
    if (!jacobi_fused) return;
    double tot = block_tree(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
    if (!last_block(&S->counter)) return;
    double g = reduce_partials(part, gridDim.x, sm);
    if (threadIdx.x == 0) cg_finalize(S, g);
}

// <r,z> + finalize when z came from a separate preconditioner apply
__global__ void k_cg_rz(int n, const double* __restrict__ r, const double* __restrict__ z, KScalars* S,
                        double* part) {
    if (S->done) return;
    __shared__ double sm[8];
    double acc = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) acc = acc + r[i] * z[i];
    }
    double tot = block_tree(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
    if (!last_block(&S->counter)) return;
    double g = reduce_partials(part, gridDim.x, sm);
    if (threadIdx.x == 0) cg_finalize(S, g);
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
__global__ void k_bicg_start(int n, const double* __restrict__ c, const double* __restrict__ r, double* p,
                             KScalars* S, double* part0, double* part1) {
    __shared__ double sm[8];
    double a0 = 0.0, a1 = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) {
            double ri = r[i];
            p[i] = ri;
            a0 = a0 + ri * ri;
            a1 = a1 + c[i] * ri;
        }
    }
    double t0 = block_tree(a0, sm);
    double t1 = block_tree(a1, sm);
    if (threadIdx.x == 0) {
        part0[blockIdx.x] = t0;
        part1[blockIdx.x] = t1;
    }
    if (!last_block(&S->counter)) return;
    double rr = reduce_partials(part0, gridDim.x, sm);
    double cr = reduce_partials(part1, gridDim.x, sm);
    if (threadIdx.x == 0) {
        double rNorm = sqrt(rr);
        S->rNorm = rNorm;
        S->iter = 0;
        S->done = 0;
        S->status = KS_RUNNING;
        if (rNorm == 0.0) {
            S->done = 1;
            S->status = KS_ZERO_RHS;
            return;
        }
        S->eps = S->atol + S->rtol * rNorm;
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

// alpha = rho / <c,v> (rho = next_rho; iteration counter advances)
__global__ void k_bicg_alpha(int n, const double* __restrict__ c, const double* __restrict__ v, KScalars* S,
                             double* part) {
    if (S->done) return;
    __shared__ double sm[8];
    double acc = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) acc = acc + c[i] * v[i];
    }
    double tot = block_tree(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
    if (!last_block(&S->counter)) return;
    double cv = reduce_partials(part, gridDim.x, sm);
    if (threadIdx.x == 0) {
        S->iter = S->iter + 1;
        S->rho = S->next_rho;
        S->cv = cv;
        S->alpha = S->rho / cv;
    }
}

// s = r - alpha v; x = x + alpha p
__global__ void k_bicg_s(int n, const double* __restrict__ r, const double* __restrict__ v,
                         const double* __restrict__ p, double* s, double* x, const KScalars* S) {
    if (S->done) return;
    double alpha = S->alpha;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) {
            s[i] = r[i] + (-alpha) * v[i];
            x[i] = x[i] + alpha * p[i];
        }
    }
}

// omega = <t,s> / <t,t>
__global__ void k_bicg_omega(int n, const double* __restrict__ t, const double* __restrict__ s, KScalars* S,
                             double* part0, double* part1) {
    if (S->done) return;
    __shared__ double sm[8];
    double a0 = 0.0, a1 = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) {
            double ti = t[i];
            a0 = a0 + ti * s[i];
            a1 = a1 + ti * ti;
        }
    }
    double t0 = block_tree(a0, sm);
    double t1 = block_tree(a1, sm);
    if (threadIdx.x == 0) {
        part0[blockIdx.x] = t0;
        part1[blockIdx.x] = t1;
    }
    if (!last_block(&S->counter)) return;
    double ts = reduce_partials(part0, gridDim.x, sm);
    double tt = reduce_partials(part1, gridDim.x, sm);
    if (threadIdx.x == 0) S->omega = ts / tt;
}

// x = x + omega s; r = s - omega t; next_rho = <c,r>; ||r||; stopping tests
__global__ void k_bicg_xr(int n, double* x, const double* __restrict__ s, const double* __restrict__ t, double* r,
                          const double* __restrict__ c, KScalars* S, double* part0, double* part1) {
    if (S->done) return;
    __shared__ double sm[8];
    double omega = S->omega;
    double a0 = 0.0, a1 = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) {
            double si = s[i];
            x[i] = x[i] + omega * si;
            double ri = si + (-omega) * t[i];
            r[i] = ri;
            a0 = a0 + c[i] * ri;
            a1 = a1 + ri * ri;
        }
    }
    double t0 = block_tree(a0, sm);
    double t1 = block_tree(a1, sm);
    if (threadIdx.x == 0) {
        part0[blockIdx.x] = t0;
        part1[blockIdx.x] = t1;
    }
    if (!last_block(&S->counter)) return;
    double cr = reduce_partials(part0, gridDim.x, sm);
    double rr = reduce_partials(part1, gridDim.x, sm);
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

// p = r + beta (p - omega v)
__global__ void k_bicg_p(int n, const double* __restrict__ r, const double* __restrict__ v, double* p,
                         const KScalars* S) {
    if (S->done) return;
    double beta = S->beta, omega = S->omega;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) p[i] = r[i] + beta * (p[i] + (-omega) * v[i]);
    }
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
    int i = rows[t];
    int ds = A.diag[i];
    double d = nz[ds];
    for (int e = row_base(A, i); e < ds; e += SELL_C) {
        int j = A.colval[e];
        d = d - (nz[A.trans[e]] * nz[e]) / D[j];
    }
    D[i] = d;
}

// forward_substitution! (preconditioners_1_DILU.jl:84-98), one level
__global__ void k_dilu_fwd(const int* __restrict__ rows, int nrows, CSRView A, const double* __restrict__ nz,
                           const double* __restrict__ D, const double* __restrict__ b, double* y,
                           const KScalars* S) {
    if (S && S->done) return;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows) return;
    int i = rows[t];
    int ds = A.diag[i];
    double sum = 0.0;
    for (int e = row_base(A, i); e < ds; e += SELL_C) {
        int j = ld_stream(A.colval + e);
        sum = sum + (ld_stream(nz + e) * y[j]) * (1.0 / D[j]);
    }
    y[i] = b[i] - sum;
}

// backward_substitution! (preconditioners_1_DILU.jl:100-114), one level, in place
__global__ void k_dilu_bwd(const int* __restrict__ rows, int nrows, CSRView A, const double* __restrict__ nz,
                           const double* __restrict__ D, double* x, const KScalars* S) {
    if (S && S->done) return;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows) return;
    int i = rows[t];
    int ds = A.diag[i];
    double sum = 0.0;
    int e1 = row_base(A, i) + SELL_C * A.len[i];
    for (int e = ds + SELL_C; e < e1; e += SELL_C) sum = sum + ld_stream(nz + e) * x[ld_stream(A.colval + e)];
    x[i] = (x[i] - sum) / D[i];
}

// residual (src/Solve/Solve_1_api.jl:441-464): ||b - A x|| / max(||b||, 1 if tiny)
__global__ void __launch_bounds__(RED_THREADS, 8) k_residual(CSRView A, const double* __restrict__ nz,
                                                          const double* __restrict__ x, const double* __restrict__ b,
                                                          KScalars* S, double* part0, double* part1, double* out) {
    __shared__ double sm[8];
    __shared__ SpmvSmem ssm;
    tile_spmv(A, nz, x, ssm);
    double a0 = 0.0, a1 = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < A.n) {
            double fx = tile_q(ssm, k);
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
// launchers
// ---------------------------------------------------------------------------
static inline int tiles(int n) { return n <= 0 ? 1 : (n + RED_TILE - 1) / RED_TILE; }
#define TILE_LAUNCH(n) tiles(n), RED_THREADS, 0

void kr_init_resid(cudaStream_t s, const CSRView& A, const double* nz, const double* b, const double* field,
                   double* dx, double* x, double* r) {
    k_init_resid<<<TILE_LAUNCH(A.n), s>>>(A, nz, b, field, dx, x, r);
    XCAL_CHECK_LAUNCH();
}
void kr_spmv(cudaStream_t s, const CSRView& A, const double* nz, const double* x, double* y, const KScalars* S) {
    k_spmv<<<TILE_LAUNCH(A.n), s>>>(A, nz, x, y, S);
    XCAL_CHECK_LAUNCH();
}
void kr_jacobi_apply(cudaStream_t s, int n, const double* P, const double* r, double* z, const KScalars* S) {
    k_jacobi_apply<<<TILE_LAUNCH(n), s>>>(n, P, r, z, S);
    XCAL_CHECK_LAUNCH();
}
void kr_copy(cudaStream_t s, int n, const double* a, double* b, const KScalars* S) {
    k_copy<<<TILE_LAUNCH(n), s>>>(n, a, b, S);
    XCAL_CHECK_LAUNCH();
}
void kr_cg_start(cudaStream_t s, int n, const double* r, const double* z, double* p, KScalars* S, double* part) {
    k_cg_start<<<TILE_LAUNCH(n), s>>>(n, r, z, p, S, part);
    XCAL_CHECK_LAUNCH();
}
void kr_cg_spmv(cudaStream_t s, const CSRView& A, const double* nz, const double* z, double* P0, double* P1,
                double* q, KScalars* S, double* part) {
    k_cg_spmv<<<TILE_LAUNCH(A.n), s>>>(A, nz, z, P0, P1, q, S, part);
    XCAL_CHECK_LAUNCH();
}
void kr_cg_update(cudaStream_t s, int n, double* x, const double* P0, const double* P1, double* r, const double* q,
                  double* z, const double* P, int jacobi_fused, KScalars* S, double* part) {
    k_cg_update<<<TILE_LAUNCH(n), s>>>(n, x, P0, P1, r, q, z, P, jacobi_fused, S, part);
    XCAL_CHECK_LAUNCH();
}
void kr_cg_rz(cudaStream_t s, int n, const double* r, const double* z, KScalars* S, double* part) {
    k_cg_rz<<<TILE_LAUNCH(n), s>>>(n, r, z, S, part);
    XCAL_CHECK_LAUNCH();
}
void kr_finish(cudaStream_t s, int n, const double* x, const double* dx, double* field) {
    k_finish<<<TILE_LAUNCH(n), s>>>(n, x, dx, field);
    XCAL_CHECK_LAUNCH();
}
void kr_bicg_start(cudaStream_t s, int n, const double* c, const double* r, double* p, KScalars* S, double* part0,
                   double* part1) {
    k_bicg_start<<<TILE_LAUNCH(n), s>>>(n, c, r, p, S, part0, part1);
    XCAL_CHECK_LAUNCH();
}
void kr_bicg_alpha(cudaStream_t s, int n, const double* c, const double* v, KScalars* S, double* part) {
    k_bicg_alpha<<<TILE_LAUNCH(n), s>>>(n, c, v, S, part);
    XCAL_CHECK_LAUNCH();
}
void kr_bicg_s(cudaStream_t s_, int n, const double* r, const double* v, const double* p, double* s, double* x,
               const KScalars* S) {
    k_bicg_s<<<TILE_LAUNCH(n), s_>>>(n, r, v, p, s, x, S);
    XCAL_CHECK_LAUNCH();
}
void kr_bicg_omega(cudaStream_t s_, int n, const double* t, const double* s, KScalars* S, double* part0,
                   double* part1) {
    k_bicg_omega<<<TILE_LAUNCH(n), s_>>>(n, t, s, S, part0, part1);
    XCAL_CHECK_LAUNCH();
}
void kr_bicg_xr(cudaStream_t s_, int n, double* x, const double* s, const double* t, double* r, const double* c,
                KScalars* S, double* part0, double* part1) {
    k_bicg_xr<<<TILE_LAUNCH(n), s_>>>(n, x, s, t, r, c, S, part0, part1);
    XCAL_CHECK_LAUNCH();
}
void kr_bicg_p(cudaStream_t s, int n, const double* r, const double* v, double* p, const KScalars* S) {
    k_bicg_p<<<TILE_LAUNCH(n), s>>>(n, r, v, p, S);
    XCAL_CHECK_LAUNCH();
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
void kr_dilu_fwd(cudaStream_t s, const int* rows, int nrows, const CSRView& A, const double* nz, const double* D,
                 const double* b, double* y, const KScalars* S) {
    if (nrows <= 0) return;
    k_dilu_fwd<<<(nrows + 255) / 256, 256, 0, s>>>(rows, nrows, A, nz, D, b, y, S);
    XCAL_CHECK_LAUNCH();
}
void kr_dilu_bwd(cudaStream_t s, const int* rows, int nrows, const CSRView& A, const double* nz, const double* D,
                 double* x, const KScalars* S) {
    if (nrows <= 0) return;
    k_dilu_bwd<<<(nrows + 255) / 256, 256, 0, s>>>(rows, nrows, A, nz, D, x, S);
    XCAL_CHECK_LAUNCH();
}
void kr_residual(cudaStream_t s, const CSRView& A, const double* nz, const double* x, const double* b, KScalars* S,
                 double* part0, double* part1, double* out) {
    k_residual<<<TILE_LAUNCH(A.n), s>>>(A, nz, x, b, S, part0, part1, out);
    XCAL_CHECK_LAUNCH();
}

}  // namespace xcal
