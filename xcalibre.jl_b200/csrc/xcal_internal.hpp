// xcal_internal.hpp -- internal structures of libxcal_b200 (host + device).
//
// Data layout in HBM (structure of arrays, int32 indices, FP64 values):
//   faces   : owner/neigh, area, delta, weight, Sf = area*normal (3), normal (3),
//             |E_f| (Laplacian non-orthogonal magnitude, internal faces)
//   cells   : volume, cell->internal-face CSR (face id, sign, CSR slot of the
//             neighbour entry), cell->boundary-face CSR (ascending face id)
//   CSR     : rowptr/colval per equation, diagonal slot per row, transpose
//             slot per entry (DILU), owner->neighbour slot per internal face
//   fields  : one array per component (vector fields component-major)
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/xcal_b200.h"
#include <nvtx3/nvToolsExt.h>

namespace xcal {

// A named NVTX range over a scope of host code (the phases of a SIMPLE
// iteration / PISO step, each equation's solve, the batch's phases), for
// timeline profilers; nvtxRangePush costs a pointer test when none is
// attached.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
struct Error {
    int code;
    std::string msg;
};

#define XCAL_CUDA(call)                                                                   \
    do {                                                                                  \
        cudaError_t _e = (call);                                                          \
        if (_e != cudaSuccess)                                                            \
            throw ::xcal::Error{_e == cudaErrorMemoryAllocation ? XCAL_ERR_OOM : XCAL_ERR_CUDA, \
                                std::string(#call) + ": " + cudaGetErrorString(_e)};     \
    } while (0)

// number of kernels this library has launched (reported by xcal_get_launch_count);
// the per-thread count lets a stream capture find how many kernels a graph holds
extern std::atomic<long long> g_launch_count;
extern thread_local long long t_launch_count;

#define XCAL_CHECK_LAUNCH()                                              \
    do {                                                                 \
        ::xcal::g_launch_count.fetch_add(1, std::memory_order_relaxed); \
        ++::xcal::t_launch_count;                                        \
        XCAL_CUDA(cudaGetLastError());                                   \
    } while (0)

inline void fail(int code, const std::string& m) { throw Error{code, m}; }

// device bytes allocated by this thread are added here while an owner (mesh
// or case under construction) has it set
extern thread_local size_t* t_alloc_acc;
struct AllocScope {  // RAII: account DBuf allocations to *acc
    size_t* prev;
    explicit AllocScope(size_t* acc) : prev(t_alloc_acc) { t_alloc_acc = acc; }
    ~AllocScope() { t_alloc_acc = prev; }
};

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        release();
        n = count;
        if (count) XCAL_CUDA(cudaMalloc(&p, count * sizeof(T)));
        if (t_alloc_acc) *t_alloc_acc += count * sizeof(T);
    }
    void zero(cudaStream_t s) {
        if (n) XCAL_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
    }
    void upload(const T* host, size_t count, cudaStream_t s) {
        alloc(count);
        if (count) XCAL_CUDA(cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T>& v, cudaStream_t s) { upload(v.data(), v.size(), s); }
};

// ---------------------------------------------------------------------------
// device views passed to kernels by value
// ---------------------------------------------------------------------------
struct MeshView {
    int nC, nF, nB;
    const int* owner;
    const int* neigh;
    const double* area;
    const double* delta;
    const double* weight;
    const double* Sx;
    const double* Sy;
    const double* Sz;
    const double* nx;
    const double* ny;
    const double* nz;
    const double* Efmag;
    const double* vol;
    const int* cf_off;
    const int* cf_face;
    const int* cf_nb;
    const signed char* cf_sign;
    const int* bf_off;   // cell -> boundary faces (ascending)
    const int* bf_face;
    const int* bcell;    // boundary_cellsID
    const int* bcells;   // list of cells that own boundary faces
    int n_bcells;
};

// Sparse matrices are stored SELL-32: rows in slices of 32 consecutive
// (storage) rows, each slice entry-major -- entry k of row r lives at
// slice[r/32] + (r%32) + 32*k -- so a warp reading entry k of its 32 rows
// issues one fully coalesced access.  Entries of a row stay in the
// reference's CSR order (ascending original column); padding entries (up to
// the slice's longest row) are never read.
constexpr int SELL_C = 32;
// systems up to this many rows apply DILU (and build its factor) in one
// block, level after level, instead of one launch per level
constexpr int DILU_BLOCK_MAX_ROWS = 65536;
// persistent CG, narrow form: prefetch a tile's matrix slots into L2 during
// the second barrier when all slots (values + columns) take at most this many
// bytes (measured: faster for a 74 MB matrix, slower for 117 and 175 MB)
constexpr long PERSIST_PF_MAX_BYTES = 80L << 20;
struct CSRView {
    int n;
    const int* slice;          // [ceil(n/32)+1] first slot of each slice
    const unsigned char* len;  // [n] entries per row
    const int* colval;
    const int* diag;   // diagonal slot per row
    const int* trans;  // slot of (col,row) per entry
    const int* cf_slot;   // slot of (cell, neighbour) per cell-face entry
    const int* fslot;     // slot of (owner, neigh) per internal face (index f - nB)
};
// slot of entry 0 of row r (entry k is at row_base + SELL_C*k)
__host__ __device__ __forceinline__ int row_base(const CSRView& A, int r) {
    return A.slice[r / SELL_C] + (r % SELL_C);
}

// per boundary face BC table of one field (U, p or nut)
struct BCView {
    const signed char* type;   // [nB] XCAL_BC_* (0 = none)
    const double* val;         // [nB*3] constant value (or DirichletFunction face values)
    // periodic (parent faces and their shadows)
    const int* peer_face;      // parent: partner face; shadow: parent face; else -1
    const int* peer_cell;      // owner of the partner face
    const double* pw;          // parent: w  (interpolation weight of own cell)
    const double* pwn;         // parent: wn (weight of the partner cell)
    const double* pEf;         // parent: |E_f| of the boundary face
    const double* pDelta;      // parent: |C2 - C1| across the periodic pair
    const double* pwdelta;     // parent: delta_p/(delta + delta_p) (rDf correction)
    const int* pNN;            // parent: CSR slot (partner cell, partner cell)
    const int* pNP;            // parent: CSR slot (partner cell, own cell)
    const int* pPN;            // parent: CSR slot (own cell, partner cell)
    // per cell: the periodic parent faces whose partner cell it is, ascending
    // ([nC+1] offsets, or null when the field has no periodic pair)
    const int* pe_off;
    const int* pe_face;
};

// per-solve device scalars (Krylov state), one 128-byte aligned block
struct alignas(128) KScalars {
    double gamma, rNorm, eps, pNorm2, alpha, beta;   // CG
    double rho, next_rho, omega, cv, resid, normb;   // BiCGSTAB / residual
    double atol, rtol;
    double rNorm0;                                    // monitored norm at the start of the solve
    // mixed precision (defect correction): outer target, inner relative
    // tolerance, outer step index, "defect already below target"
    double eps_outer, inner_rtol;
    int mixed, outer, outer_conv;
    int total;                                        // mixed: inner iterations over all outer steps
    int loops;                                        // graph mode: bodies run by the current WHILE loop
    int iter, itmax, done, status;
    unsigned int counter;                             // last-block ticket
    unsigned int counter2;
};
enum {
    KS_RUNNING = 0,
    KS_SOLVED = 1,
    KS_TIRED = 2,
    KS_ZERO_CURV = 3,
    KS_BREAKDOWN = 4,
    KS_ZERO_RHS = 5,
    KS_LOOP_CAP = 6  // graph mode: a device-driven loop hit its body-count cap
};

}  // namespace xcal
