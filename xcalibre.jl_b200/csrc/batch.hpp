// batch.hpp -- batched Krylov solves over many independent cases.
//
// A batch holds the resident cases of a request stream.  Their pressure and
// momentum systems form one block-diagonal system: each case keeps its own
// SELL matrix, vectors and Krylov scalars, and a launch covers every case at
// once through a per-system descriptor table and a tile map (block b works on
// local tile tmap[b].y of system tmap[b].x).  Row sums and reduction trees are
// the single-case ones, so a case's result does not depend on the batch it
// ran in.
#pragma once
#include "kernels.hpp"
#include "xcal_internal.hpp"

namespace xcal {

// roles of the work vectors in a batched system descriptor
enum {
    KV_X = 0,  // iterate
    KV_R,      // residual
    KV_Z,      // preconditioned residual (CG; = KV_R without preconditioner)
    KV_P,      // direction (CG p_k of even k)
    KV_Q,      // A * direction
    KV_V,      // CG p_k of odd k; BiCGSTAB v
    KV_S,      // BiCGSTAB s
    KV_T,      // BiCGSTAB t
    KV_C,      // BiCGSTAB shadow vector (right-hand side)
    KV_R0,     // BiCGSTAB unpreconditioned initial residual
    KV_COUNT
};

template <class T>
struct BSys {
    CSRView A;
    const T* nz;
    const T* P;  // Jacobi inverse diagonal or DILU D
    T* vec[KV_COUNT];
    KScalars* S;
    double* part0;
    double* part1;
    int n;
    int ntiles;
    // level-ordered triangles (one-block DILU sweeps of small systems)
    LevelView<T> lo, up;
};

// FP64 side of one equation slot of a case inside a batched solve: the
// matrix and vectors the solve's start, finish, mixed-precision defect
// correction and residual touch, and the DILU level copies to refresh
struct BAux {
    CSRView A;
    const double* nz;
    float* nz32;        // FP32 copy (mixed)
    const double* P;    // Jacobi inverse diagonal or DILU D
    float* P32;         // its FP32 copy (mixed; null: no preconditioner)
    const double* b;
    double* field;
    double* dx;         // FP64 path: warm-start shift
    double* x;          // FP64 path: Krylov iterate
    double* r0;         // FP64 path: initial residual (r for CG, q for BiCGSTAB)
    float* d32;         // mixed: defect = inner right-hand side
    float* x32;         // mixed: inner iterate
    KScalars* S;        // the case's scalars in the batch (residual counter, outer flags)
    double* part0;
    double* part1;
    double* res_out;    // scaled residual of this slot
    // DILU: level-ordered triangles (lsrc null: no DILU)
    const int* lsrc;
    const int* lcol;
    const int* lslice;
    double* lval;
    float* lval32;
    double* ldinv;
    float* ldinv32;
    const int* usrc;
    const int* uslice;
    double* uval;
    float* uval32;
    int n, ntiles;
};

// batched per-case steps of a solve (one launch over the tile map instead of
// one launch per case); the arithmetic of k_init_resid, k_finish, k_defect,
// k_correct (masked by outer_conv), k_residual, k_to_float, k_gather_vals and
// k_level_dinv
void kb_init_resid(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total);
void kb_finish(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total);
void kb_defect(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total);
void kb_correct(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total);
void kb_residual(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total);
void kb_to_float(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total);
// level copies of the DILU triangles: values from nz (fp32: nz32) and the
// lower triangle's 1/D per slot from P (fp32: P32)
void kb_level_refresh(cudaStream_t s, const BAux* aux, const int2* tmap, int ntiles_total, int fp32);

// batched launchers (kernels_batch.cu); tmap has ntiles_total entries
template <class T>
void kb_spmv(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total, int in, int out);
template <class T>
void kb_jacobi_apply(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total, int in, int out,
                     int use_S);
template <class T>
void kb_copy(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total, int in, int out, int use_S);
// DILU application: systems listed in small_ids (n <= DILU_BLOCK_MAX_ROWS)
// one block each over their level-ordered triangles (y in shared memory when
// the largest of them, small_n rows, fits), the others level by level over
// merged (system, row) lists
template <class T>
void kb_dilu(cudaStream_t s, const BSys<T>* sys, const int* small_ids, int n_small, int small_n, const int2* lo_rows,
             const std::vector<int>& lo_off, const int2* up_rows, const std::vector<int>& up_off, int in, int out,
             int use_S);
template <class T>
void kb_cg_start(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total);
// every system's CG solve (Jacobi: jacobi = 1; none: 0) in one cooperative
// launch; false (nothing launched) when the tiles cannot all be co-resident.
// bars: 2 words per system of the batch (nbars systems), err as in
// kr_cg_persist.
template <class T>
bool kb_cg_persist(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total, int jacobi,
                   unsigned int* bars, int nbars, int* err, int max_iters, int width = 0);
// the cluster form: every listed system (ids[0..nsys)) as one thread-block
// cluster of the size its largest member needs; false (nothing launched)
// when max_tiles exceeds PERSIST_CLUSTER_MAX or the device cannot run it
template <class T>
bool kb_cg_persist_cluster(cudaStream_t s, const BSys<T>* sys, const int* ids, int nsys, int max_tiles, int jacobi,
                           int max_iters);
// the cluster-form kernel (for persist_cluster_size queries)
template <class T>
const void* kb_cg_persist_cluster_kernel();
template <class T>
void kb_cg_spmv(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total);
template <class T>
void kb_cg_update(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total, int jacobi_fused);
template <class T>
void kb_cg_rz(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total);
template <class T>
void kb_bicg_start(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total);
template <class T>
void kb_bicg_alpha(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total);
template <class T>
void kb_bicg_s(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total);
template <class T>
void kb_bicg_omega(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total);
template <class T>
void kb_bicg_xr(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total);
template <class T>
void kb_bicg_p(cudaStream_t s, const BSys<T>* sys, const int2* tmap, int ntiles_total);

}  // namespace xcal
