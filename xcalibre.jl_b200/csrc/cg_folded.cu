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
// residual and the previous direction are gathered as one (r, p) pair per
// neighbour; the block's rows of x, p and q stay in shared memory for the
// whole solve (x reaches HBM only as the final FP64 correction), so HBM sees
// the matrix, the gathered pairs, and the write of each row's next pair.
//
// Launch shape: one block of 768 or 1024 threads per SM (cooperative), each
// owning a contiguous run of rows -- 148 blocks meet at each grid barrier
// instead of one per 2048-row tile.  Reductions are deterministic: every thread adds
// its rows in a fixed order (FP64 accumulators), the block adds its warps
// in a fixed tree, and every block adds the block partials in the same
// order, so every block takes the same decisions.
#include <cooperative_groups.h>

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

// every thread's value summed over the block in a fixed order, for thread
// 0 only (one block barrier; sm: 32 doubles, free again after the next
// block barrier)
__device__ __forceinline__ double fold_block_partial(double v, double* sm) {
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    double w = 0.0;
    if (warp == 0) {
        w = lane < nw ? sm[lane] : 0.0;
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) w = w + __shfl_xor_sync(0xffffffffu, w, off);
    }
    return w;
}

// the block partials of one reduction, added in the same order by every
// block: warp 0 alone (lane l adds partials l, l + 32, ... in turn, then the
// lanes' sums in a fixed tree), the total handed to the block through sm[32]
// with one block barrier
__device__ __forceinline__ double fold_grid_sum(const double* part, int nblocks, double* sm) {
    if (threadIdx.x < 32) {
        double v = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += 32) v = v + __ldcg(part + b);
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, off);
        if (threadIdx.x == 0) sm[32] = v;
    }
    __syncthreads();
    return sm[32];
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
        const double tot = fold_block_partial(acc, sm);
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
        const double tot2 = fold_block_partial(acc2, sm);
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

// launch geometry of the folded CG (form `form`) for n rows: blocks (one per
// SM while the rows fit), rows per block (a multiple of 32) and which vectors
// stay in shared memory; blocks = 0 when the system does not fit
FoldShape fold_shape(int n, int form, bool vectors_in_smem) {
    // once per process (one device type) and form: SM count, and whether a
    // block with the largest shared-memory request is co-resident on an SM
    static int sms = -1;
    static int attr_ok[FOLD_NFORMS] = {-1, -1, -1, -1};
    if (form < 0 || form >= FOLD_NFORMS) form = FOLD_DEFAULT_FORM;
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

bool kr_cgf_persist(cudaStream_t s, const FoldView& F, float2* RP0, float2* RP1, float* xg, double* field,
                    const double* Pj, KScalars* S, double* part, double* part2, unsigned int* bar, int* err,
                    int max_iters, bool reset_err, int form, bool vectors_in_smem) {
    const FoldShape sh = fold_shape(F.n, form, vectors_in_smem);
    if (sh.blocks <= 0) return false;
    XCAL_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned int), s));
    if (reset_err) XCAL_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    FoldView Fv = F;
    int R = sh.rows, sp = sh.smem_p ? 1 : 0, sx = sh.smem_x ? 1 : 0;
    void* args[] = {&Fv, &RP0, &RP1, &xg, &field, (void*)&Pj, &S, &part, &part2, &bar, &err, &max_iters,
                    &R, &sp, &sx};
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
    XCAL_CUDA(cudaLaunchKernelExC(&cfg, FOLD_FORMS[F.W > 0 ? 1 : 0][sh.form].fn, args));
    XCAL_CHECK_LAUNCH();
    return true;
}

}  // namespace xcal
