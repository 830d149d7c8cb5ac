// kernels_batch.cu -- batched Krylov kernels: one launch over the tiles of
// every system in a batch (block-diagonal system with per-system offsets).
// Each block looks up its (system, local tile) and runs the same tile body as
// the single-system kernel (krylov_bodies.cuh).
#include <vector>

#include "batch.hpp"
#include "kernels.hpp"
#include "krylov_bodies.cuh"

namespace xcal {

#define XCAL_BSYS                                   \
    const int2 tm = tmap[blockIdx.x];               \
    const BSys<T>& B = sys[tm.x];                   \
    const TileCtx tc{tm.y, B.ntiles};

template <class T>
__global__ void __launch_bounds__(RED_THREADS, 8) kbk_spmv(const BSys<T>* __restrict__ sys, const int2* tmap, int in,
                                                        int out) {
    XCAL_BSYS
    spmv_body<T>(tc, B.A, B.nz, B.vec[in], B.vec[out], B.S);
}

template <class T>
__global__ void kbk_jacobi_apply(const BSys<T>* __restrict__ sys, const int2* tmap, int in, int out, int use_S) {
    XCAL_BSYS
    jacobi_apply_body<T>(tc, B.n, B.P, B.vec[in], B.vec[out], use_S ? B.S : nullptr);
}

template <class T>
__global__ void kbk_copy(const BSys<T>* __restrict__ sys, const int2* tmap, int in, int out, int use_S) {
    XCAL_BSYS
    copy_body<T>(tc, B.n, B.vec[in], B.vec[out], use_S ? B.S : nullptr);
}

// one DILU level over the rows (system, row) of every system at that level
template <class T>
__global__ void kbk_dilu_fwd(const BSys<T>* __restrict__ sys, const int2* __restrict__ rows, int nrows, int in,
                             int out, int use_S) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows) return;
    const int2 r = rows[t];
    const BSys<T>& B = sys[r.x];
    if (use_S && B.S->done) return;
    dilu_fwd_row<T>(B.A, B.nz, B.P, B.vec[in], B.vec[out], r.y);
}

template <class T>
__global__ void kbk_dilu_bwd(const BSys<T>* __restrict__ sys, const int2* __restrict__ rows, int nrows, int out,
                             int use_S) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows) return;
    const int2 r = rows[t];
    const BSys<T>& B = sys[r.x];
    if (use_S && B.S->done) return;
    dilu_bwd_row<T>(B.A, B.nz, B.P, B.vec[out], r.y);
}

// one block per small system: a whole DILU application
template <class T>
__global__ void __launch_bounds__(DILU_BLOCK_THREADS) kbk_dilu_block(const BSys<T>* __restrict__ sys,
                                                                     const int* __restrict__ ids, int in, int out,
                                                                     int use_S, int smem) {
    extern __shared__ __align__(16) unsigned char dilu_smem[];
    const BSys<T>& B = sys[ids[blockIdx.x]];
    if (use_S && B.S->done) return;
    T* y = B.vec[out];
    dilu_level_sweep<T>(B.n, B.lo, B.up, B.P, B.vec[in], y, smem ? reinterpret_cast<T*>(dilu_smem) : y);
}

template <class T>
__global__ void kbk_cg_start(const BSys<T>* __restrict__ sys, const int2* tmap) {
    XCAL_BSYS
    cg_start_body<T>(tc, B.n, B.vec[KV_R], B.vec[KV_Z], B.vec[KV_P], B.S, B.part0);
}

template <class T>
__global__ void __launch_bounds__(RED_THREADS, 8) kbk_cg_spmv(const BSys<T>* __restrict__ sys, const int2* tmap) {
    XCAL_BSYS
    cg_spmv_body<T>(tc, B.A, B.nz, B.vec[KV_Z], B.vec[KV_P], B.vec[KV_V], B.vec[KV_Q], B.S, B.part0);
}

template <class T>
__global__ void __launch_bounds__(RED_THREADS, sizeof(T) == 4 ? 4 : 8) kbk_cg_update(const BSys<T>* __restrict__ sys, const int2* tmap, int jacobi_fused) {
    XCAL_BSYS
    cg_update_body<T>(tc, B.n, B.vec[KV_X], B.vec[KV_P], B.vec[KV_V], B.vec[KV_R], B.vec[KV_Q], B.vec[KV_Z], B.P,
                      jacobi_fused, B.S, B.part0);
}

template <class T>
__global__ void kbk_cg_rz(const BSys<T>* __restrict__ sys, const int2* tmap) {
    XCAL_BSYS
    cg_rz_body<T>(tc, B.n, B.vec[KV_R], B.vec[KV_Z], B.S, B.part0);
}

template <class T>
__global__ void kbk_bicg_start(const BSys<T>* __restrict__ sys, const int2* tmap) {
    XCAL_BSYS
    bicg_start_body<T>(tc, B.n, B.vec[KV_C], B.vec[KV_R], B.vec[KV_P], B.S, B.part0, B.part1);
}

template <class T>
__global__ void kbk_bicg_alpha(const BSys<T>* __restrict__ sys, const int2* tmap) {
    XCAL_BSYS
    bicg_alpha_body<T>(tc, B.n, B.vec[KV_C], B.vec[KV_V], B.S, B.part0);
}

template <class T>
__global__ void kbk_bicg_s(const BSys<T>* __restrict__ sys, const int2* tmap) {
    XCAL_BSYS
    bicg_s_body<T>(tc, B.n, B.vec[KV_R], B.vec[KV_V], B.vec[KV_P], B.vec[KV_S], B.vec[KV_X], B.S);
}

template <class T>
__global__ void kbk_bicg_omega(const BSys<T>* __restrict__ sys, const int2* tmap) {
    XCAL_BSYS
    bicg_omega_body<T>(tc, B.n, B.vec[KV_T], B.vec[KV_S], B.S, B.part0, B.part1);
}

template <class T>
__global__ void kbk_bicg_xr(const BSys<T>* __restrict__ sys, const int2* tmap) {
    XCAL_BSYS
    bicg_xr_body<T>(tc, B.n, B.vec[KV_X], B.vec[KV_S], B.vec[KV_T], B.vec[KV_R], B.vec[KV_C], B.S, B.part0,
                    B.part1);
}

template <class T>
__global__ void kbk_bicg_p(const BSys<T>* __restrict__ sys, const int2* tmap) {
    XCAL_BSYS
    bicg_p_body<T>(tc, B.n, B.vec[KV_R], B.vec[KV_V], B.vec[KV_P], B.S);
}

// every system's whole CG solve in one cooperative launch: the blocks of a
// system synchronise only among themselves (barrier state bars[2 s .. 2 s+1]),
// so systems finish independently
template <class T, int NT>
__global__ void __launch_bounds__(NT, persist_min_blocks(NT))
    kbk_cg_persist(const BSys<T>* __restrict__ sys, const int2* tmap, int jacobi, unsigned int* bars, int* err,
                   int max_iters) {
    XCAL_BSYS
    cg_persist_body<T, NT>(tc, B.A, B.nz, B.P, jacobi, B.vec[KV_X], B.vec[KV_R], B.vec[KV_Z], B.vec[KV_P],
                           B.vec[KV_V], B.S, B.part0, B.part1, bars + 2 * tm.x, err, max_iters, 0);
}

// cluster form: system ids[b / C] is the cluster of blocks b (rank b % C)
template <class T>
__global__ void __launch_bounds__(1024, 1) kbk_cg_persist_cl(const BSys<T>* __restrict__ sys,
                                                            const int* __restrict__ ids, int C, int jacobi,
                                                            int max_iters) {
    const BSys<T>& B = sys[ids[blockIdx.x / C]];
    const TileCtx tc{(int)(blockIdx.x % C), B.ntiles};
    cg_persist_body<T, 1024, true>(tc, B.A, B.nz, B.P, jacobi, B.vec[KV_X], B.vec[KV_R], B.vec[KV_Z], B.vec[KV_P],
                                   B.vec[KV_V], B.S, nullptr, nullptr, nullptr, nullptr, max_iters, 0);
}

// ---- per-case steps of a solve, batched (BAux tables) ----
#define XCAL_BAUX                                   \
    const int2 tm = tmap[blockIdx.x];               \
    const BAux& B = aux[tm.x];                      \
    const TileCtx tc{tm.y, B.ntiles};

// r0 = b - A field, x = 0, dx = field (k_init_resid)
__global__ void __launch_bounds__(RED_THREADS, 8) kbx_init_resid(const BAux* __restrict__ aux, const int2* tmap) {
    XCAL_BAUX
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < B.n) {
            B.r0[i] = B.b[i] - row_dot(B.A, B.nz, (const double*)B.field, i);
            B.x[i] = 0.0;
            B.dx[i] = B.field[i];
        }
    }
}

// field = x + dx (k_finish)
__global__ void kbx_finish(const BAux* __restrict__ aux, const int2* tmap) {
    XCAL_BAUX
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < B.n) B.field[i] = B.x[i] + B.dx[i];
    }
}

// d32 = (float)(b - A field), x32 = 0 (k_defect)
__global__ void __launch_bounds__(RED_THREADS, 8) kbx_defect(const BAux* __restrict__ aux, const int2* tmap) {
    XCAL_BAUX
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < B.n) {
            B.d32[i] = (float)(B.b[i] - row_dot(B.A, B.nz, (const double*)B.field, i));
            B.x32[i] = 0.0f;
        }
    }
}

// field += x32 unless the outer loop found the defect already at its target
// (k_correct; the case then leaves the outer loop uncorrected)
__global__ void kbx_correct(const BAux* __restrict__ aux, const int2* tmap) {
    XCAL_BAUX
    if (B.S->outer_conv) return;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < B.n) B.field[i] = B.field[i] + (double)B.x32[i];
    }
}

// ||b - A field|| / max(||b||, 1 if tiny) per system (k_residual: the same
// tile trees, the last of the system's blocks finishes)
__global__ void __launch_bounds__(RED_THREADS, 8) kbx_residual(const BAux* __restrict__ aux, const int2* tmap) {
    XCAL_BAUX
    __shared__ double sm[8];
    double a0 = 0.0, a1 = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(tc, k);
        if (i < B.n) {
            double fx = row_dot(B.A, B.nz, (const double*)B.field, i);
            double bi = B.b[i];
            double d = bi - fx;
            a0 = a0 + d * d;
            a1 = a1 + bi * bi;
        }
    }
    double t0 = block_tree(a0, sm);
    double t1 = block_tree(a1, sm);
    if (threadIdx.x == 0) {
        B.part0[tc.tile] = t0;
        B.part1[tc.tile] = t1;
    }
    if (!last_block(&B.S->counter2, tc.ntiles)) return;
    double sR = reduce_partials(B.part0, tc.ntiles, sm);
    double sb = reduce_partials(B.part1, tc.ntiles, sm);
    if (threadIdx.x == 0) {
        double normb = sqrt(sb);
        double denom = normb > jl_eps(normb) ? normb : 1.0;
        double res = sqrt(sR) / denom;
        B.S->resid = res;
        B.S->normb = normb;
        *B.res_out = res;
    }
}

// nz32 = (float) nz over the tile's slots (its rows' slices are contiguous),
// P32 = (float) P over its rows
__global__ void kbx_to_float(const BAux* __restrict__ aux, const int2* tmap) {
    XCAL_BAUX
    const int s0 = tc.tile * (RED_TILE / SELL_C);
    const int s1 = min(s0 + RED_TILE / SELL_C, (B.n + SELL_C - 1) / SELL_C);
    const int e1 = B.A.slice[s1];
    for (int e = B.A.slice[s0] + threadIdx.x; e < e1; e += blockDim.x) B.nz32[e] = (float)ld_stream(B.nz + e);
    if (B.P32)
        for (int k = 0; k < RED_ITEMS; ++k) {
            int i = tile_row(tc, k);
            if (i < B.n) B.P32[i] = (float)B.P[i];
        }
}

// level copies: slots of level positions in the tile (contiguous slices)
template <class T>
__device__ __forceinline__ void level_refresh_tile(const TileCtx& tc, int n, const int* slice, const int* src,
                                                   const T* nz, T* val, const int* col, const T* D, T* dinv) {
    const int s0 = tc.tile * (RED_TILE / SELL_C);
    const int s1 = min(s0 + RED_TILE / SELL_C, (n + SELL_C - 1) / SELL_C);
    const int e1 = slice[s1];
    for (int e = slice[s0] + threadIdx.x; e < e1; e += blockDim.x) {
        val[e] = nz[ld_stream(src + e)];
        if (dinv) dinv[e] = T(1) / D[ld_stream(col + e)];
    }
}

__global__ void kbx_level_refresh(const BAux* __restrict__ aux, const int2* tmap, int fp32) {
    XCAL_BAUX
    if (!B.lsrc) return;
    if (fp32) {
        level_refresh_tile<float>(tc, B.n, B.lslice, B.lsrc, B.nz32, B.lval32, B.lcol, B.P32, B.ldinv32);
        level_refresh_tile<float>(tc, B.n, B.uslice, B.usrc, B.nz32, B.uval32, nullptr, nullptr, nullptr);
    } else {
        level_refresh_tile<double>(tc, B.n, B.lslice, B.lsrc, B.nz, B.lval, B.lcol, B.P, B.ldinv);
        level_refresh_tile<double>(tc, B.n, B.uslice, B.usrc, B.nz, B.uval, nullptr, nullptr, nullptr);
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
#define XCAL_XLAUNCH(K, ...)                                     \
    do {                                                         \
        if (ntiles_total <= 0) return;                           \
        K<<<ntiles_total, RED_THREADS, 0, s>>>(__VA_ARGS__);     \
        XCAL_CHECK_LAUNCH();                                     \
    } while (0)
void kb_init_resid(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total) {
    XCAL_XLAUNCH(kbx_init_resid, aux, tmap);
}
void kb_finish(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total) {
    XCAL_XLAUNCH(kbx_finish, aux, tmap);
}
void kb_defect(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total) {
    XCAL_XLAUNCH(kbx_defect, aux, tmap);
}
void kb_correct(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total) {
    XCAL_XLAUNCH(kbx_correct, aux, tmap);
}
void kb_residual(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total) {
    XCAL_XLAUNCH(kbx_residual, aux, tmap);
}
void kb_to_float(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total) {
    XCAL_XLAUNCH(kbx_to_float, aux, tmap);
}
void kb_level_refresh(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total, int fp32) {
    XCAL_XLAUNCH(kbx_level_refresh, aux, tmap, fp32);
}
#define XCAL_BLAUNCH(K, ...)                                     \
    do {                                                         \
        if (ntiles_total <= 0) return;                           \
        K<T><<<ntiles_total, RED_THREADS, 0, s>>>(__VA_ARGS__);  \
        XCAL_CHECK_LAUNCH();                                     \
    } while (0)

template <class T>
void kb_spmv(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total, int in, int out) {
    XCAL_BLAUNCH(kbk_spmv, sys, tmap, in, out);
}
template <class T>
void kb_jacobi_apply(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total, int in, int out,
                     int use_S) {
    XCAL_BLAUNCH(kbk_jacobi_apply, sys, tmap, in, out, use_S);
}
template <class T>
void kb_copy(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total, int in, int out, int use_S) {
    XCAL_BLAUNCH(kbk_copy, sys, tmap, in, out, use_S);
}
template <class T>
void kb_dilu(cudaStream_t s, const BSys<T>* sys, const int* small_ids, int n_small, int small_n, const int2* lo_rows,
             const std::vector<int>& lo_off, const int2* up_rows, const std::vector<int>& up_off, int in, int out,
             int use_S) {
    if (n_small > 0) {
        static bool attr_set = false;
        if (!attr_set) {
            XCAL_CUDA(cudaFuncSetAttribute(kbk_dilu_block<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           DILU_SMEM_MAX_BYTES));
            attr_set = true;
        }
        const size_t bytes = (size_t)small_n * sizeof(T);
        const int smem = bytes <= (size_t)DILU_SMEM_MAX_BYTES ? 1 : 0;
        kbk_dilu_block<T><<<n_small, DILU_BLOCK_THREADS, smem ? bytes : 0, s>>>(sys, small_ids, in, out, use_S, smem);
        XCAL_CHECK_LAUNCH();
    }
    for (size_t l = 0; l + 1 < lo_off.size(); ++l) {
        int nr = lo_off[l + 1] - lo_off[l];
        if (nr <= 0) continue;
        kbk_dilu_fwd<T><<<(nr + 255) / 256, 256, 0, s>>>(sys, lo_rows + lo_off[l], nr, in, out, use_S);
        XCAL_CHECK_LAUNCH();
    }
    for (size_t l = 0; l + 1 < up_off.size(); ++l) {
        int nr = up_off[l + 1] - up_off[l];
        if (nr <= 0) continue;
        kbk_dilu_bwd<T><<<(nr + 255) / 256, 256, 0, s>>>(sys, up_rows + up_off[l], nr, out, use_S);
        XCAL_CHECK_LAUNCH();
    }
}
template <class T>
bool kb_cg_persist(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total, int jacobi,
                   unsigned int* bars, int nbars, int* err, int max_iters, int width) {
    static PersistCaps caps;
    static const void* const kern[3] = {(const void*)kbk_cg_persist<T, 1024>, (const void*)kbk_cg_persist<T, 512>,
                                        (const void*)kbk_cg_persist<T, RED_THREADS>};
    const int w = persist_pick(caps, kern, ntiles_total, width);
    if (w < 0) return false;
    XCAL_CUDA(cudaMemsetAsync(bars, 0, 2 * (size_t)nbars * sizeof(unsigned int), s));
    XCAL_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    void* args[] = {(void*)&sys, (void*)&tmap, &jacobi, &bars, &err, &max_iters};
    return persist_launch(caps, w, kern[w], ntiles_total, s, args);
}
template <class T>
const void* kb_cg_persist_cluster_kernel() {
    return (const void*)kbk_cg_persist_cl<T>;
}
template <class T>
bool kb_cg_persist_cluster(cudaStream_t s, const BSys<T>* sys, const int* ids, int nsys, int max_tiles, int jacobi,
                           int max_iters) {
    const void* k = (const void*)kbk_cg_persist_cl<T>;
    const int C = persist_cluster_size(k, max_tiles);
    if (C == 0 || nsys <= 0) return false;
    int Cv = C;
    void* args[] = {(void*)&sys, (void*)&ids, &Cv, &jacobi, &max_iters};
    persist_cluster_launch(k, C, nsys, s, args);
    return true;
}
template <class T>
void kb_cg_start(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total) {
    XCAL_BLAUNCH(kbk_cg_start, sys, tmap);
}
template <class T>
void kb_cg_spmv(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total) {
    XCAL_BLAUNCH(kbk_cg_spmv, sys, tmap);
}
template <class T>
void kb_cg_update(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total, int jacobi_fused) {
    XCAL_BLAUNCH(kbk_cg_update, sys, tmap, jacobi_fused);
}
template <class T>
void kb_cg_rz(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total) {
    XCAL_BLAUNCH(kbk_cg_rz, sys, tmap);
}
template <class T>
void kb_bicg_start(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total) {
    XCAL_BLAUNCH(kbk_bicg_start, sys, tmap);
}
template <class T>
void kb_bicg_alpha(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total) {
    XCAL_BLAUNCH(kbk_bicg_alpha, sys, tmap);
}
template <class T>
void kb_bicg_s(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total) {
    XCAL_BLAUNCH(kbk_bicg_s, sys, tmap);
}
template <class T>
void kb_bicg_omega(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total) {
    XCAL_BLAUNCH(kbk_bicg_omega, sys, tmap);
}
template <class T>
void kb_bicg_xr(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total) {
    XCAL_BLAUNCH(kbk_bicg_xr, sys, tmap);
}
template <class T>
void kb_bicg_p(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total) {
    XCAL_BLAUNCH(kbk_bicg_p, sys, tmap);
}

#define XCAL_BATCH_INSTANTIATE(T)                                                                                 \
    template void kb_spmv<T>(cudaStream_t, const BSys<T>*, const int2*, int, int, int);                            \
    template void kb_jacobi_apply<T>(cudaStream_t, const BSys<T>*, const int2*, int, int, int, int);               \
    template void kb_copy<T>(cudaStream_t, const BSys<T>*, const int2*, int, int, int, int);                       \
    template void kb_dilu<T>(cudaStream_t, const BSys<T>*, const int*, int, int, const int2*,                    \
                             const std::vector<int>&,                                                             \
                             const int2*, const std::vector<int>&, int, int, int);                                \
    template void kb_cg_start<T>(cudaStream_t, const BSys<T>*, const int2*, int);                                  \
    template bool kb_cg_persist<T>(cudaStream_t, const BSys<T>*, const int2*, int, int, unsigned int*, int, int*,  \
                                   int, int);                                                                     \
    template bool kb_cg_persist_cluster<T>(cudaStream_t, const BSys<T>*, const int*, int, int, int, int);          \
    template const void* kb_cg_persist_cluster_kernel<T>();                                                         \
    template void kb_cg_spmv<T>(cudaStream_t, const BSys<T>*, const int2*, int);                                   \
    template void kb_cg_update<T>(cudaStream_t, const BSys<T>*, const int2*, int, int);                            \
    template void kb_cg_rz<T>(cudaStream_t, const BSys<T>*, const int2*, int);                                     \
    template void kb_bicg_start<T>(cudaStream_t, const BSys<T>*, const int2*, int);                                \
    template void kb_bicg_alpha<T>(cudaStream_t, const BSys<T>*, const int2*, int);                                \
    template void kb_bicg_s<T>(cudaStream_t, const BSys<T>*, const int2*, int);                                    \
    template void kb_bicg_omega<T>(cudaStream_t, const BSys<T>*, const int2*, int);                                \
    template void kb_bicg_xr<T>(cudaStream_t, const BSys<T>*, const int2*, int);                                   \
    template void kb_bicg_p<T>(cudaStream_t, const BSys<T>*, const int2*, int);
XCAL_BATCH_INSTANTIATE(double)
XCAL_BATCH_INSTANTIATE(float)

}  // namespace xcal
