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

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
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
