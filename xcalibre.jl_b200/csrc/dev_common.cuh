// dev_common.cuh -- device helpers shared by the kernels.
//
// Arithmetic contract (matches the reference's Julia code, which never fuses
// a*b+c): the library is compiled with --fmad=false, every expression below
// is written in the operation order of the cited Julia source, and all
// reductions use the fixed "canonical tile" tree so results are
// deterministic and independent of scheduling.
#pragma once
#include <cuda_runtime.h>

#include "xcal_internal.hpp"

namespace xcal {

// canonical reduction geometry: a tile is RED_THREADS threads x RED_ITEMS rows;
// thread t of tile b owns rows b*RED_TILE + k*RED_THREADS + t, k < RED_ITEMS
constexpr int RED_THREADS = 256;
constexpr int RED_ITEMS = 8;
constexpr int RED_TILE = RED_THREADS * RED_ITEMS;

__device__ __forceinline__ int tile_row(int k) { return blockIdx.x * RED_TILE + k * RED_THREADS + threadIdx.x; }

// The tile a block works on and the number of tiles of its system: the grid
// itself for a single system; a (system, local tile) map entry for a batched
// launch over many independent systems (block-diagonal, per-system offsets).
struct TileCtx {
    int tile;
    int ntiles;
};
__device__ __forceinline__ TileCtx grid_tiles() { return TileCtx{(int)blockIdx.x, (int)gridDim.x}; }
__device__ __forceinline__ int tile_row(const TileCtx& tc, int k) {
    return tc.tile * RED_TILE + k * RED_THREADS + threadIdx.x;
}

// Load of data read once per launch (matrix slots, vectors consumed by their
// last reader): evict-first in L1 and L2, so the streams do not push the
// gathered vectors out of L2.  Measured on the 2M-cell pressure matrix: the
// CG SpMV drops from 59 to 53 us.
template <class T>
__device__ __forceinline__ T ld_stream(const T* p) { return __ldcs(p); }

// Julia's max(x, y) for floats (NaN propagating, -0.0 < 0.0)
__device__ __forceinline__ double jl_max(double x, double y) {
    bool take_y = (y > x) || (signbit(y) < signbit(x));
    return take_y ? (isnan(x) ? x : y) : (isnan(y) ? y : x);
}

// Julia's min(x, y) for floats (NaN propagating, -0.0 < 0.0)
__device__ __forceinline__ double jl_min(double x, double y) {
    bool take_y = (y < x) || (signbit(y) > signbit(x));
    return take_y ? (isnan(x) ? x : y) : (isnan(y) ? y : x);
}

// exp(y) for y <= 0 and tanh(x) for x >= 0 from +, *, / and ldexp only, the
// same operations on the host and the device: Cody-Waite reduction
// y = k ln2 + r (ln2 split in a 12-bit head and its remainder), exp(r) by its
// Taylor series to r^14 / 14!; tanh(x) = (1 - e^-2x) / (1 + e^-2x), 1 past 20
__host__ __device__ __forceinline__ double det_exp_neg(double y) {
    if (y < -745.0) return 0.0;
    const double LN2_HEAD = 0.693145751953125, LN2_TAIL = 1.4286068203094172321e-06;
    const double k = rint(y * 1.4426950408889634);
    const double r = (y - k * LN2_HEAD) - k * LN2_TAIL;
    double p = 1.0;
    for (int n = 14; n >= 1; --n) p = 1.0 + (r / (double)n) * p;
    return ldexp(p, (int)k);
}
// log(x) for x > 0 from frexp (exact) and +, *, /: x = 2^e m with
// m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s), s = (m - 1) / (m + 1), by
// its series to s^29
__host__ __device__ __forceinline__ double det_log(double x) {
    int e = 0;
    double m = frexp(x, &e);
    if (m < 0.70710678118654752) {
        m = 2.0 * m;
        e -= 1;
    }
    const double s = (m - 1.0) / (m + 1.0), s2 = s * s;
    double t = 0.0;
    for (int n = 29; n >= 3; n -= 2) t = (t + 1.0 / (double)n) * s2;
    return (double)e * 0.6931471805599453 + 2.0 * (s + s * t);
}
__host__ __device__ __forceinline__ double det_tanh_pos(double x) {
    if (x > 20.0) return 1.0;
    const double e = det_exp_neg(-2.0 * x);
    return (1.0 - e) / (1.0 + e);
}
// x^a for x >= 0 as exp(a log x) (k-omega LKE's Re_upsilon^-1.30): 0^a =
// Inf for a < 0, Inf^a = 0; det_exp_neg's reduction also holds for y > 0,
// up to the overflow at 709.7
__host__ __device__ __forceinline__ double det_pow(double x, double a) {
    if (x == 0.0) return a < 0.0 ? INFINITY : 0.0;
    if (isinf(x)) return a < 0.0 ? 0.0 : INFINITY;
    const double y = a * det_log(x);
    return y >= 709.7 ? INFINITY : det_exp_neg(y);
}

// Julia's eps(x)
__device__ __forceinline__ double jl_eps(double x) {
    x = fabs(x);
    return nextafter(x, __longlong_as_double(0x7ff0000000000000ULL)) - x;
}

// Block tree of the canonical reduction: xor butterfly (16..1) inside each
// warp, then butterfly (4,2,1) over the 8 warp sums.  Result valid in thread 0.
// In blocks wider than RED_THREADS (the persistent CG's wide form) only
// threads 0..RED_THREADS-1 contribute; every thread must call it.
__device__ __forceinline__ double block_tree(double v, double* smem8) {
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();  // smem8 may still be read by a previous tree
    if (lane == 0 && warp < RED_THREADS / 32) smem8[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
        double w = lane < (RED_THREADS / 32) ? smem8[lane] : 0.0;
#pragma unroll
        for (int off = (RED_THREADS / 64); off >= 1; off >>= 1) w = w + __shfl_xor_sync(0xffffffffu, w, off);
        r = w;
    }
    return r;
}

// Final pass over tile partials (executed by one block): thread t sums
// partials t, t+RED_THREADS, ... sequentially, then the block tree.
__device__ __forceinline__ double reduce_partials(const double* part, int T, double* smem8) {
    double s = 0.0;
    if (threadIdx.x < RED_THREADS)
        for (int i = threadIdx.x; i < T; i += RED_THREADS) s = s + __ldcg(part + i);
    return block_tree(s, smem8);
}

// Last-block election among the ntiles blocks of one system: every block
// publishes its partial(s) before calling; returns true in all threads of the
// block that arrives last (the counter is reset by it).  No block waits, so
// there is no spin.
__device__ __forceinline__ bool last_block(unsigned int* counter, int ntiles) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int ticket = atomicAdd(counter, 1u);
        is_last = (ticket == (unsigned int)ntiles - 1u);
        if (is_last) *counter = 0u;
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}
__device__ __forceinline__ bool last_block(unsigned int* counter) { return last_block(counter, (int)gridDim.x); }

}  // namespace xcal
