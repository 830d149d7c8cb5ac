// cg_folded.cu -- the FP32 inner CG of mixed precision, on the Jacobi-scaled
// system.
//
// Krylov.jl's cg! with the Jacobi preconditioner M = diag(1/|a_ii|) applied
// by multiplication (Solve_1_api.jl:268-307, preconditioners_2_functions.jl:
// 65-98) is, in exact arithmetic, plain CG on
//     Ahat = M^1/2 A M^1/2,   rhat = M^1/2 r,   x = M^1/2 xhat:
// every scalar of the iteration is the same (<r, z> = <rhat, rhat>,
// <p, A p> = <phat, Ahat phat>, so alpha, beta, the monitored norm
// sqrt(<r, z>) and the stopping tests coincide).  Ahat has +-1 on its
// diagonal, so only its off-diagonal entries are stored and z = M r
// disappears.  This form is used for the FP32 inner solves of the FP64
// defect correction, whose contract is a tolerance against the FP64 path,
// not bit-exactness with it; the FP64 path keeps the canonical kernel.
//
// Per iteration the off-diagonal slots (value + column) stream once; the
// direction and residual are gathered; the block's rows of x, p and q stay
// in shared memory for the whole solve (x reaches HBM only as the final FP64
// correction), so HBM sees the matrix, two gathered vectors, and the writes
// of p and r.
//
// Launch shape: one 1024-thread block per SM (cooperative), each owning a
// contiguous run of rows -- 148 blocks meet at each grid barrier instead of
// one per 2048-row tile.  Reductions are deterministic: every thread adds
// its rows in a fixed order (FP64 accumulators), the block adds its warps
// in a fixed tree, and every block adds the block partials in the same
// order, so every block takes the same decisions.
#include <cooperative_groups.h>

#include <algorithm>
#include <vector>

#include "dev_common.cuh"
#include "kernels.hpp"
#include "krylov_bodies.cuh"

namespace xcal {

// dynamic shared memory per block (q, then p and x when they fit)
constexpr int FOLD_SMEM_MAX = 220 * 1024;

// rp[i].x = r_i = (float)(sqrt(P_i) (b_i - sum_j a_ij field_j)) -- the
// scaled FP64 defect (row sums in the row's CSR order, FP64)
__global__ void __launch_bounds__(RED_THREADS, 8) k_fold_defect(CSRView A, const double* __restrict__ nz,
                                                             const double* __restrict__ b,
                                                             const double* __restrict__ field,
                                                             const double* __restrict__ P, float2* rp) {
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < A.n) rp[i].x = (float)(sqrt(P[i]) * (b[i] - row_dot(A, nz, field, i)));
    }
}

// start of the inner solve: gamma = <r, r> over rp[].x (canonical tile
// tree, the last block finishing), then cg!'s start tests (cg_start_scalars)
__global__ void __launch_bounds__(RED_THREADS) k_fold_start(int n, const float2* __restrict__ rp, KScalars* S,
                                                            double* part) {
    __shared__ double sm[8];
    double acc = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        const int i = tile_row(k);
        if (i < n) {
            const double ri = (double)rp[i].x;
            acc = acc + ri * ri;
        }
    }
    const double tot = block_tree(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
    if (!last_block(&S->counter)) return;
    const double gamma = reduce_partials(part, (int)gridDim.x, sm);
    if (threadIdx.x == 0) cg_start_scalars(S, gamma);
}

// scaled off-diagonal values ahat_ij = a_ij sqrt(P_i) sqrt(P_j) (FP64, then
// rounded), and the sign of each row's diagonal in bit 7 of its length byte
__global__ void k_fold_scale(int n, const int* __restrict__ slice, unsigned char* len, const int* __restrict__ col,
                             const int* __restrict__ map, float* val, const double* __restrict__ nz,
                             const int* __restrict__ diag, const double* __restrict__ P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double si = sqrt(P[i]);
    const int base = slice[i >> 5] + (i & 31);
    const int ln = len[i] & 0x7f;
    for (int m = 0; m < ln; ++m) {
        const int s = base + SELL_C * m;
        val[s] = (float)((nz[map[s]] * si) * sqrt(P[col[s]]));
    }
    len[i] = (unsigned char)(ln | (nz[diag[i]] < 0.0 ? 0x80 : 0));
}

// every thread's value summed over the block in a fixed order; valid in
// every thread (sm: 33 doubles)
__device__ __forceinline__ double fold_block_sum(double v, double* sm) {
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();  // sm may still be read by the previous sum
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double w = lane < nw ? sm[lane] : 0.0;
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) w = w + __shfl_xor_sync(0xffffffffu, w, off);
        if (lane == 0) sm[32] = w;
    }
    __syncthreads();
    return sm[32];
}

// the block partials of one reduction, added in the same order by every block
__device__ __forceinline__ double fold_grid_sum(const double* part, int nblocks, double* sm) {
    double v = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v = v + __ldcg(part + b);
    return fold_block_sum(v, sm);
}

// The first U off-diagonal slots of a row (columns and values), loaded
// together.  UNI (every slice padded to the same width W, padding slots
// holding the row's own column and a zero value): the row's first slot sits
// at 32 W (i / 32) + i % 32, so no slice offset and no row length stand in
// front of these loads; else the slice offset and the row length are read
// first and only the row's own slots are loaded.
template <int U>
struct FoldSlots {
    int c[U];
    float v[U];
};
template <bool UNI, int U>
__device__ __forceinline__ void fold_load(const FoldView& F, int i, FoldSlots<U>& s) {
    if constexpr (UNI) {
        const int base = SELL_C * F.W * (i >> 5) + (i & 31);
#pragma unroll
        for (int m = 0; m < U; ++m)
            if (m < F.W) {
                s.c[m] = ld_stream(F.col + base + SELL_C * m);
                s.v[m] = ld_stream(F.val + base + SELL_C * m);
            }
    } else {
        const int ln = F.len[i] & 0x7f;
        const int base = F.slice[i >> 5] + (i & 31);
#pragma unroll
        for (int m = 0; m < U; ++m)
            if (m < ln) {
                s.c[m] = ld_stream(F.col + base + SELL_C * m);
                s.v[m] = ld_stream(F.val + base + SELL_C * m);
            }
    }
}

// q_i = s_i d_i + sum_j ahat_ij d_j over row i's off-diagonal slots (s_i the
// sign of its diagonal), with d = r (first iteration: p_0 = z = r) or
// r + beta p_old, formed for every gathered column the same way; slots past
// the first U are read here
// d_j = r_j (first iteration) or r_j + beta p_old_j, from one 8-byte load of
// the pair (r_j, p_old_j)
template <bool FIRST>
__device__ __forceinline__ float fold_dir(const float2* rp, float beta, int j) {
    const float2 g = rp[j];
    return FIRST ? g.x : __fmaf_rn(beta, g.y, g.x);
}

// q_i = s_i d_i + sum_j ahat_ij d_j over row i's off-diagonal slots (s_i the
// sign of its diagonal), every d formed the same way (fold_dir); rp = the
// current pairs (r, p_old); slots past the first U are read here
template <bool FIRST, bool UNI, int U>
__device__ __forceinline__ float fold_q(const FoldView& F, const float2* rp, float beta, int i,
                                        const FoldSlots<U>& s, float& pi) {
    const unsigned lb = F.len[i];
    const int n_slots = UNI ? F.W : (int)(lb & 0x7f);
    pi = fold_dir<FIRST>(rp, beta, i);
    float q = (lb & 0x80) ? -pi : pi;
#pragma unroll
    for (int m = 0; m < U; ++m)
        if (m < n_slots) q = __fmaf_rn(s.v[m], fold_dir<FIRST>(rp, beta, s.c[m]), q);
    if (n_slots > U) {
        const int base = UNI ? SELL_C * F.W * (i >> 5) + (i & 31) : F.slice[i >> 5] + (i & 31);
        for (int m = U; m < n_slots; ++m) {
            const int sl = base + SELL_C * m;
            q = __fmaf_rn(ld_stream(F.val + sl), fold_dir<FIRST>(rp, beta, ld_stream(F.col + sl)), q);
        }
    }
    return q;
}

// The whole inner solve (Krylov.jl cg! in the scaled variables) in one
// cooperative launch.  Entered after k_fold_start: the scalar block holds
// gamma = <rhat, rhat>, eps and the stopping state, RP0[].x = rhat.  The
// residual and the previous direction travel as pairs (r_i, p_old_i) in two
// buffers that swap every iteration (cur = RP0 on even iterations): a
// neighbour's direction value r_j + beta p_old_j is one 8-byte load.
// Per iteration
//   phase 1: p_k (gathered neighbours formed on the fly from cur), q = Ahat
//            p_k into shared memory, block partial of <p_k, q>;
//   barrier; alpha (same value in every block), zero-curvature test;
//   phase 2: x += alpha p_k (shared memory), nxt_i = (r_i - alpha q_i, p_k,i),
//            partial <r, r>;
//   barrier; cg! stopping tests, beta.
// At the end, unless the defect already met the outer target (outer_conv),
// field_i += sqrt(P_i) xhat_i in FP64: the correction of this defect step.
// Block 0 writes the scalar state back.  smem_x / smem_p: x / p_k kept in
// shared memory (else in xg / nxt[].y, stored in phase 1).
//
// NT threads per block; U slots per row issued together (the rest in a
// loop); PIPE: a thread issues the slot loads of its next row before it
// gathers for the current one, so the two rows' loads overlap.  UNI: the
// uniform-width slot layout (fold_load).  Each row's arithmetic is the same
// in every shape; only the grouping of the block partials follows NT.
template <int NT, int U, bool PIPE, bool UNI>
__global__ void __launch_bounds__(NT, 1)
    k_cgf_persist(FoldView F, float2* RP0, float2* RP1, float* xg, double* field, const double* __restrict__ Pj,
                  KScalars* S, double* part, double* part2, unsigned int* bar, int* err, int max_iters, int R,
                  int smem_p, int smem_x) {
    extern __shared__ float fold_sm[];
    __shared__ double sm[33];
    __shared__ int sh_err;
    float* q_s = fold_sm;
    float* p_s = fold_sm + R;
    float* x_s = fold_sm + (smem_p ? 2 * R : R);
    const int n = F.n;
    const int row0 = blockIdx.x * R;
    const int nr = max(0, min(R, n - row0));
    const int G = gridDim.x;
    for (int k = threadIdx.x; k < nr; k += NT) {
        if (smem_x)
            x_s[k] = 0.0f;
        else
            xg[row0 + k] = 0.0f;
    }
    int iter = S->iter, done = S->done, status = S->status;
    const int itmax = S->itmax, outer_conv = S->outer_conv;
    double gamma = S->gamma, beta = S->beta, pNorm2 = S->pNorm2, alpha = S->alpha, rNorm = S->rNorm;
    const double eps = S->eps;
    const double epsT = 1.1920928955078125e-07;  // eps(Float32)
    unsigned int nb = 0;
    bool ok = true;
    int ran = 0;
    while (!done && ran < max_iters) {
        const float2* cur = (iter & 1) ? RP1 : RP0;
        float2* nxt = (iter & 1) ? RP0 : RP1;
        const float bt = (float)beta;
        double acc = 0.0;
        FoldSlots<U> sl, sl_next;
        int k = threadIdx.x;
        if (PIPE && k < nr) fold_load<UNI, U>(F, row0 + k, sl);
        for (; k < nr; k += NT) {
            const int i = row0 + k;
            if constexpr (PIPE) {
                if (k + NT < nr) fold_load<UNI, U>(F, i + NT, sl_next);
            } else {
                fold_load<UNI, U>(F, i, sl);
            }
            float pi, qi;
            if (iter == 0)
                qi = fold_q<true, UNI, U>(F, cur, bt, i, sl, pi);
            else
                qi = fold_q<false, UNI, U>(F, cur, bt, i, sl, pi);
            q_s[k] = qi;
            if (smem_p)
                p_s[k] = pi;
            else
                nxt[i].y = pi;
            acc = acc + (double)pi * (double)qi;
            if constexpr (PIPE) sl = sl_next;
        }
        double tot = fold_block_sum(acc, sm);
        if (threadIdx.x == 0) part[blockIdx.x] = tot;
        if (!(ok = grid_barrier(bar, G, nb, err, &sh_err))) break;
        const double pAp = fold_grid_sum(part, G, sm);
        const double lim = epsT * pNorm2;
        if (pAp <= lim && fabs(pAp) <= lim) {
            done = 1;
            status = KS_ZERO_CURV;
            break;
        }
        alpha = gamma / pAp;
        const float a = (float)alpha;
        double acc2 = 0.0;
        for (int k = threadIdx.x; k < nr; k += NT) {
            const int i = row0 + k;
            const float pi = smem_p ? p_s[k] : nxt[i].y;
            if (smem_x)
                x_s[k] = __fmaf_rn(a, pi, x_s[k]);
            else
                xg[i] = __fmaf_rn(a, pi, xg[i]);
            const float ri = __fmaf_rn(-a, q_s[k], cur[i].x);
            nxt[i] = make_float2(ri, pi);
            acc2 = acc2 + (double)ri * (double)ri;
        }
        double tot2 = fold_block_sum(acc2, sm);
        if (threadIdx.x == 0) part2[blockIdx.x] = tot2;
        if (!(ok = grid_barrier(bar, G, nb, err, &sh_err))) break;
        const double g = fold_grid_sum(part2, G, sm);
        // cg! stopping tests (the same as cg_finalize), in every thread
        rNorm = sqrt(g);
        const bool solved = (rNorm <= eps) || (rNorm + 1.0 <= 1.0);
        if (!solved) {
            const double b2 = g / gamma;
            pNorm2 = g + (b2 * b2) * pNorm2;
            gamma = g;
            beta = b2;
        }
        iter = iter + 1;
        if (solved) {
            done = 1;
            status = KS_SOLVED;
        } else if (iter >= itmax) {
            done = 1;
            status = KS_TIRED;
        }
        ++ran;
    }
    if (!ok) return;
    if (!outer_conv)
        for (int k = threadIdx.x; k < nr; k += NT) {
            const int i = row0 + k;
            const float xh = smem_x ? x_s[k] : xg[i];
            field[i] = field[i] + sqrt(Pj[i]) * (double)xh;
        }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
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

// ---------------------------------------------------------------------------
// Staged form: the matrix slots reach shared memory by bulk asynchronous
// copies (cp.async.bulk, completion counted on an mbarrier), so no slot load
// stands in front of a row's gathers and the copy engine, not the warps'
// registers, keeps the matrix stream in flight.  Uniform slot layout only.
//
// Each warp owns a ring of `nstage` stages; a stage holds one slice (32
// rows): W columns, W values and the 32 length bytes, 256 W + 32 bytes.  A
// warp's slices are the ones its rows fall in (rows 32 (w + j NW) + lane of
// the block, exactly the rows the other forms give that thread), taken in
// order, then again from the first: the matrix does not change during the
// solve, so the copies of the next iteration's first slices run during the
// grid barriers.  A stage is refilled as soon as the warp has used it.
//
// Per row the arithmetic is fold_q's, and the rows each thread adds are the
// same as in k_cgf_persist with the same NT: the two give the same results
// bit for bit.  p_k is not stored: phase 2 re-forms it from the same pair
// (r, p_old) with the same operation.  Every wait is bounded; a stage wait
// that gives up sets the error flag and the block leaves before the next
// grid barrier (the others then leave theirs); copies still in flight are
// waited for, with the same bound, before any block exits.

constexpr int STAGE_WMAX = 8;             // widest uniform row (slots) the staged form takes
constexpr int STAGE_MAX = 6;              // stages per warp at most
constexpr int STAGE_SMEM_MAX = 224 * 1024;  // dynamic shared memory (q, x, stages)
constexpr long STAGE_SPIN_LIMIT = 1L << 24;  // polls before a stage wait gives up

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned long long* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_done(unsigned long long* b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for the completion of phase `parity`; false: gave up
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity) {
    for (long k = 0; k < STAGE_SPIN_LIMIT; ++k)
        if (mbar_done(b, parity)) return true;
    return false;
}
// global -> this block's shared memory, `bytes` (a multiple of 16, both
// addresses 16-byte aligned), counted on b
__device__ __forceinline__ void bulk_to_smem(void* dst, const void* src, unsigned bytes, unsigned long long* b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(b))
                 : "memory");
}

// q_i and p_i of row i from its slots, already read out of the stage (c,
// v: columns and values; lb: the row's length byte)
template <bool FIRST>
__device__ __forceinline__ float stage_q(const float2* rp, float beta, int i, int W, const int (&c)[STAGE_WMAX],
                                         const float (&v)[STAGE_WMAX], unsigned lb, float& pi) {
    pi = fold_dir<FIRST>(rp, beta, i);
    float q = (lb & 0x80) ? -pi : pi;
#pragma unroll
    for (int m = 0; m < STAGE_WMAX; ++m)
        if (m < W) q = __fmaf_rn(v[m], fold_dir<FIRST>(rp, beta, c[m]), q);
    return q;
}

template <int NT>
__global__ void __launch_bounds__(NT, 1)
    k_cgf_staged(FoldView F, float2* RP0, float2* RP1, float* xg, double* field, const double* __restrict__ Pj,
                 KScalars* S, double* part, double* part2, unsigned int* bar, int* err, int max_iters, int R,
                 int smem_x, int nstage) {
    constexpr int NW = NT / 32;
    extern __shared__ __align__(128) unsigned char stage_raw[];
    __shared__ double sm[33];
    __shared__ int sh_err, sh_stage;
    __shared__ unsigned long long mbar[NW * STAGE_MAX];
    const int W = F.W;
    const int SB = 256 * W + 32;  // bytes of one stage
    float* q_s = (float*)stage_raw;
    float* x_s = q_s + R;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* ring = stage_raw + 4L * R * (1 + smem_x) + (long)warp * nstage * SB;
    unsigned long long* wb = mbar + warp * STAGE_MAX;
    const int n = F.n;
    const int row0 = blockIdx.x * R;
    const int nr = max(0, min(R, n - row0));
    const int G = gridDim.x;
    // this warp's slices per iteration (local slice j: rows 32 (warp + j NW) + lane)
    const int nsw = nr > 32 * warp ? (nr - 32 * warp + 32 * NW - 1) / (32 * NW) : 0;
    if (threadIdx.x == 0) sh_stage = 0;
    if (lane == 0)
        for (int s = 0; s < nstage; ++s) mbar_init(wb + s, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncthreads();
    // this warp's stage sequence (the same in every lane): the next stage
    // to fill and the local slice it gets; the next stage to use and the
    // parity of the fill it waits for; fills not yet used
    int iss_s = 0, iss_j = 0, use_s = 0, pending = 0;
    unsigned use_ph = 0;
    auto issue = [&]() {
        if (lane == 0) {
            const long g = (long)(row0 >> 5) + warp + (long)iss_j * NW;
            unsigned char* st = ring + (long)iss_s * SB;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect(wb + iss_s, (unsigned)SB);
            bulk_to_smem(st, F.col + (long)SELL_C * W * g, 128u * W, wb + iss_s);
            bulk_to_smem(st + 128 * W, F.val + (long)SELL_C * W * g, 128u * W, wb + iss_s);
            bulk_to_smem(st + 256 * W, F.len + (long)SELL_C * g, 32u, wb + iss_s);
        }
        iss_s = iss_s + 1 == nstage ? 0 : iss_s + 1;
        iss_j = iss_j + 1 == nsw ? 0 : iss_j + 1;
        ++pending;
    };
    auto retire = [&]() {
        if (++use_s == nstage) {
            use_s = 0;
            use_ph ^= 1u;
        }
        --pending;
    };
    if (nsw > 0)
        for (int s = 0; s < nstage; ++s) issue();
    for (int k = threadIdx.x; k < nr; k += NT) {
        if (smem_x)
            x_s[k] = 0.0f;
        else
            xg[row0 + k] = 0.0f;
    }
    int iter = S->iter, done = S->done, status = S->status;
    const int itmax = S->itmax, outer_conv = S->outer_conv;
    double gamma = S->gamma, beta = S->beta, pNorm2 = S->pNorm2, alpha = S->alpha, rNorm = S->rNorm;
    const double eps = S->eps;
    const double epsT = 1.1920928955078125e-07;  // eps(Float32)
    unsigned int nb = 0;
    bool ok = true;
    int ran = 0;
    while (!done && ran < max_iters) {
        const float2* cur = (iter & 1) ? RP1 : RP0;
        float2* nxt = (iter & 1) ? RP0 : RP1;
        const float bt = (float)beta;
        double acc = 0.0;
        for (int j = 0; j < nsw; ++j) {
            if (!__all_sync(0xffffffffu, mbar_wait(wb + use_s, use_ph))) {
                if (lane == 0) sh_stage = 1;
                break;
            }
            // read the row's slots out of the stage, then refill the stage
            // before the gathers, so the copy runs while they wait
            const unsigned char* st = ring + (long)use_s * SB;
            const int k = SELL_C * (warp + j * NW) + lane;
            int c[STAGE_WMAX];
            float v[STAGE_WMAX];
            unsigned lb = 0;
            if (k < nr) {
                const int* cs = (const int*)st;
                const float* vs = (const float*)(st + 128 * W);
#pragma unroll
                for (int m = 0; m < STAGE_WMAX; ++m)
                    if (m < W) {
                        c[m] = cs[SELL_C * m + lane];
                        v[m] = vs[SELL_C * m + lane];
                    }
                lb = st[256 * W + lane];
            }
            __syncwarp();
            retire();
            issue();
            if (k < nr) {
                const int i = row0 + k;
                float pi, qi;
                if (iter == 0)
                    qi = stage_q<true>(cur, bt, i, W, c, v, lb, pi);
                else
                    qi = stage_q<false>(cur, bt, i, W, c, v, lb, pi);
                q_s[k] = qi;
                acc = acc + (double)pi * (double)qi;
            }
        }
        double tot = fold_block_sum(acc, sm);
        if (sh_stage) {  // uniform: read after the block sum's barriers
            if (threadIdx.x == 0) *(volatile int*)err = 1;
            ok = false;
            break;
        }
        if (threadIdx.x == 0) part[blockIdx.x] = tot;
        if (!(ok = grid_barrier(bar, G, nb, err, &sh_err))) break;
        const double pAp = fold_grid_sum(part, G, sm);
        const double lim = epsT * pNorm2;
        if (pAp <= lim && fabs(pAp) <= lim) {
            done = 1;
            status = KS_ZERO_CURV;
            break;
        }
        alpha = gamma / pAp;
        const float a = (float)alpha;
        double acc2 = 0.0;
        for (int k = threadIdx.x; k < nr; k += NT) {
            const int i = row0 + k;
            const float2 g = cur[i];
            const float pi = iter == 0 ? g.x : __fmaf_rn(bt, g.y, g.x);
            if (smem_x)
                x_s[k] = __fmaf_rn(a, pi, x_s[k]);
            else
                xg[i] = __fmaf_rn(a, pi, xg[i]);
            const float ri = __fmaf_rn(-a, q_s[k], g.x);
            nxt[i] = make_float2(ri, pi);
            acc2 = acc2 + (double)ri * (double)ri;
        }
        double tot2 = fold_block_sum(acc2, sm);
        if (threadIdx.x == 0) part2[blockIdx.x] = tot2;
        if (!(ok = grid_barrier(bar, G, nb, err, &sh_err))) break;
        const double g2 = fold_grid_sum(part2, G, sm);
        // cg! stopping tests (the same as cg_finalize), in every thread
        rNorm = sqrt(g2);
        const bool solved = (rNorm <= eps) || (rNorm + 1.0 <= 1.0);
        if (!solved) {
            const double b2 = g2 / gamma;
            pNorm2 = g2 + (b2 * b2) * pNorm2;
            gamma = g2;
            beta = b2;
        }
        iter = iter + 1;
        if (solved) {
            done = 1;
            status = KS_SOLVED;
        } else if (iter >= itmax) {
            done = 1;
            status = KS_TIRED;
        }
        ++ran;
    }
    // the copies still in flight land before the block's shared memory goes
    while (pending > 0) {
        mbar_wait(wb + use_s, use_ph);
        retire();
    }
    __syncwarp();
    if (!ok) return;
    if (!outer_conv)
        for (int k = threadIdx.x; k < nr; k += NT) {
            const int i = row0 + k;
            const float xh = smem_x ? x_s[k] : xg[i];
            field[i] = field[i] + sqrt(Pj[i]) * (double)xh;
        }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
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

void kr_fold_defect(cudaStream_t s, const CSRView& A, const double* nz, const double* b, const double* field,
                    const double* P, float2* rp) {
    k_fold_defect<<<(A.n + RED_TILE - 1) / RED_TILE, RED_THREADS, 0, s>>>(A, nz, b, field, P, rp);
    XCAL_CHECK_LAUNCH();
}

void kr_fold_start(cudaStream_t s, int n, const float2* rp, KScalars* S, double* part) {
    k_fold_start<<<(n + RED_TILE - 1) / RED_TILE, RED_THREADS, 0, s>>>(n, rp, S, part);
    XCAL_CHECK_LAUNCH();
}

void kr_fold_scale(cudaStream_t s, const FoldMut& F, const double* nz, const int* diag, const double* P) {
    k_fold_scale<<<(F.n + 255) / 256, 256, 0, s>>>(F.n, F.slice, F.len, F.col, F.map, F.val, nz, diag, P);
    XCAL_CHECK_LAUNCH();
}

// the kernel forms (threads per block, slots per row issued together, row
// pairs), selected by index
struct FoldKernel {
    const void* fn;
    int nt;
};
static const FoldKernel FOLD_FORMS[2][FOLD_NFORMS] = {
    {
        {(const void*)k_cgf_persist<768, 6, false, false>, 768},
        {(const void*)k_cgf_persist<1024, 6, false, false>, 1024},
        {(const void*)k_cgf_persist<768, 6, true, false>, 768},
        {(const void*)k_cgf_persist<1024, 6, true, false>, 1024},
    },
    {
        {(const void*)k_cgf_persist<768, 6, false, true>, 768},
        {(const void*)k_cgf_persist<1024, 6, false, true>, 1024},
        {(const void*)k_cgf_persist<768, 6, true, true>, 768},
        {(const void*)k_cgf_persist<1024, 6, true, true>, 1024},
    },
};

// the staged forms (index form - FOLD_NFORMS): uniform slot layout only
static const FoldKernel STAGED[FOLD_NSTAGED] = {
    {(const void*)k_cgf_staged<768>, 768},
    {(const void*)k_cgf_staged<1024>, 1024},
};

// launch geometry of the folded CG (form `form`) for n rows: blocks (one per
// SM while the rows fit), rows per block (a multiple of 32) and which vectors
// stay in shared memory; blocks = 0 when the system does not fit
FoldShape fold_shape(int n, int form, bool vectors_in_smem) {
    // once per process (one device type) and form: SM count, and whether a
    // block with the largest shared-memory request is co-resident on an SM
    static int sms = -1;
    static int attr_ok[FOLD_NFORMS] = {-1, -1, -1, -1};
    if (form < 0 || form >= FOLD_NFORMS + FOLD_NSTAGED) form = FOLD_DEFAULT_FORM;
    if (form >= FOLD_NFORMS) {
        // a staged form: the blocks and rows of the pipelined form with its
        // thread count (its fallback when the staged geometry does not fit)
        FoldShape sh = fold_shape(n, form - 2, vectors_in_smem);
        if (sh.blocks > 0) sh.form = form;
        return sh;
    }
    if (sms < 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            sms = 0;
        cudaGetLastError();
    }
    if (attr_ok[form] < 0) {
        attr_ok[form] = 1;
        for (int uni = 0; uni < 2; ++uni) {  // both slot layouts of the form
            int per = 0;
            const FoldKernel& K = FOLD_FORMS[uni][form];
            if (cudaFuncSetAttribute(K.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, FOLD_SMEM_MAX) !=
                    cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, K.fn, K.nt, FOLD_SMEM_MAX) != cudaSuccess ||
                per < 1)
                attr_ok[form] = 0;
        }
        cudaGetLastError();
    }
    FoldShape sh;
    if (sms <= 0 || attr_ok[form] != 1 || n <= 0) return sh;
    int R = (n + sms - 1) / sms;
    R = (R + SELL_C - 1) / SELL_C * SELL_C;
    const long q = 4L * R;
    if (q > FOLD_SMEM_MAX) return sh;
    if ((n + R - 1) / R > FOLD_MAX_BLOCKS) return sh;
    sh.form = form;
    sh.nt = FOLD_FORMS[0][form].nt;
    sh.blocks = (n + R - 1) / R;
    sh.rows = R;
    sh.smem_p = vectors_in_smem && 2 * q <= FOLD_SMEM_MAX;
    sh.smem_x = vectors_in_smem && (sh.smem_p ? 3 : 2) * q <= FOLD_SMEM_MAX;
    sh.smem = (int)(q * (1 + sh.smem_p + sh.smem_x));
    return sh;
}

// geometry of a staged form for rows of W slots: stages per warp and
// whether x stays in shared memory; false when it does not fit (the caller
// then runs the pipelined form with the same thread count)
static bool stage_shape(const FoldShape& sh, int W, bool vectors_in_smem, int& nstage, int& smem_x, int& smem) {
    if (W <= 0 || W > STAGE_WMAX) return false;
    const int k = sh.form - FOLD_NFORMS;
    static int attr_ok[FOLD_NSTAGED] = {-1, -1};
    if (attr_ok[k] < 0) {
        int per = 0;
        attr_ok[k] = cudaFuncSetAttribute(STAGED[k].fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          STAGE_SMEM_MAX) == cudaSuccess &&
                     cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, STAGED[k].fn, STAGED[k].nt,
                                                                   STAGE_SMEM_MAX) == cudaSuccess &&
                     per >= 1;
        cudaGetLastError();
    }
    if (attr_ok[k] != 1) return false;
    const long per_stage = (long)(STAGED[k].nt / 32) * (256L * W + 32);
    for (int sx = vectors_in_smem ? 1 : 0; sx >= 0; --sx) {
        const long vec = 4L * sh.rows * (1 + sx);
        const long ns = std::min<long>(STAGE_MAX, (STAGE_SMEM_MAX - vec) / per_stage);
        if (ns >= 2) {
            nstage = (int)ns;
            smem_x = sx;
            smem = (int)(vec + ns * per_stage);
            return true;
        }
    }
    return false;
}

bool kr_cgf_persist(cudaStream_t s, const FoldView& F, float2* RP0, float2* RP1, float* xg, double* field,
                    const double* Pj, KScalars* S, double* part, double* part2, unsigned int* bar, int* err,
                    int max_iters, bool reset_err, int form, bool vectors_in_smem) {
    FoldShape sh = fold_shape(F.n, form, vectors_in_smem);
    if (sh.blocks <= 0) return false;
    XCAL_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned int), s));
    if (reset_err) XCAL_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    FoldView Fv = F;
    int R = sh.rows, sp = sh.smem_p ? 1 : 0, sx = sh.smem_x ? 1 : 0;
    int nstage = 0, ssx = 0, ssmem = 0;
    const void* fn = nullptr;
    std::vector<void*> args;
    if (sh.form >= FOLD_NFORMS) {
        if (stage_shape(sh, F.W, vectors_in_smem, nstage, ssx, ssmem)) {
            fn = STAGED[sh.form - FOLD_NFORMS].fn;
            args = {&Fv, &RP0, &RP1, &xg, &field, (void*)&Pj, &S, &part, &part2, &bar, &err, &max_iters,
                    &R, &ssx, &nstage};
            sh.smem = ssmem;
        } else {
            sh = fold_shape(F.n, sh.form - 2, vectors_in_smem);
            sp = sh.smem_p ? 1 : 0;
            sx = sh.smem_x ? 1 : 0;
        }
    }
    if (!fn) {
        fn = FOLD_FORMS[F.W > 0 ? 1 : 0][sh.form].fn;
        args = {&Fv, &RP0, &RP1, &xg, &field, (void*)&Pj, &S, &part, &part2, &bar, &err, &max_iters,
                &R, &sp, &sx};
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(sh.blocks);
    cfg.blockDim = dim3(sh.nt);
    cfg.dynamicSmemBytes = sh.smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    XCAL_CUDA(cudaLaunchKernelExC(&cfg, fn, args.data()));
    XCAL_CHECK_LAUNCH();
    return true;
}

}  // namespace xcal
