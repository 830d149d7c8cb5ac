// noalloc.cu -- scaled CSR residual without any device allocation.
//
// Some callers cannot call cudaMalloc: code running while a CUDA graph is
// being captured, hosts that hand the library a fixed memory budget or a
// stream-ordered pool they manage themselves, or a Julia task holding the
// GPU under a no-allocation policy.  xcal_residual_noalloc serves them: the
// caller passes the CSR arrays, x, b and a device pointer for the result, all
// already in device memory, and the library uses only the fixed scratch array
// below for its reduction (tile partials and the last-block counter).
//
// The array is a file-scope __device__ variable, so every GPU that loads the
// library holds it (NOALLOC_BYTES, about 256 KiB) until the process exits.
// All calls share it and it keeps the previous call's contents: the counter
// that must start at zero is cleared by every call, and calls whose work
// overlaps on the GPU (different streams, or different host threads on the
// same device) race on it -- callers serialise them.
#include <mutex>

#include "dev_common.cuh"

namespace xcal {

constexpr int NOALLOC_MAX_ROWS = 1 << 25;                   // 33,554,432 rows
constexpr int NOALLOC_MAX_TILES = NOALLOC_MAX_ROWS / RED_TILE;  // 16,384
constexpr size_t NOALLOC_HDR = 256;                         // counter, padded
constexpr size_t NOALLOC_BYTES = NOALLOC_HDR + 2 * sizeof(double) * NOALLOC_MAX_TILES;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

// Same arithmetic as the residual that ends solve_system! (k_residual):
// per-row sum in CSR order, canonical tile trees for sum((b-Ax)^2) and
// sum(b^2), denominator ||b|| unless it is at most eps(||b||).
__global__ void __launch_bounds__(RED_THREADS) k_residual_noalloc(int n, const int* __restrict__ rowptr,
                                                                  const int* __restrict__ colval,
                                                                  const double* __restrict__ nz,
                                                                  const double* __restrict__ x,
                                                                  const double* __restrict__ b,
                                                                  unsigned char* scratch, double* result) {
    __shared__ double sm[8];
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch);
    double* part0 = reinterpret_cast<double*>(scratch + NOALLOC_HDR);
    double* part1 = part0 + NOALLOC_MAX_TILES;
    double a0 = 0.0, a1 = 0.0;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) {
            double fx = 0.0;
            for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) fx = fx + nz[e] * x[colval[e]];
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
    if (!last_block(counter)) return;
    double sR = reduce_partials(part0, gridDim.x, sm);
    double sb = reduce_partials(part1, gridDim.x, sm);
    if (threadIdx.x == 0) {
        double normb = sqrt(sb);
        double denom = normb > jl_eps(normb) ? normb : 1.0;
        *result = sqrt(sR) / denom;
    }
}

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[256] = {nullptr};

void set_msg(char* err, int errlen, const char* msg) {
    if (!err || errlen <= 0) return;
    int i = 0;
    for (; msg[i] && i < errlen - 1; ++i) err[i] = msg[i];
    err[i] = 0;
}
}  // namespace

}  // namespace xcal

using namespace xcal;

extern "C" int32_t xcal_residual_noalloc(int32_t n, const int32_t* rowptr, const int32_t* colval,
                                         const double* nzval, const double* x, const double* b,
                                         double* result, void* stream, char* err, int32_t errlen) {
    if (n <= 0 || n > NOALLOC_MAX_ROWS) {
        set_msg(err, errlen, "xcal_residual_noalloc: n must be in 1..33554432 (the fixed scratch holds 16384 tiles)");
        return XCAL_ERR_INVALID;
    }
    if (!rowptr || !colval || !nzval || !x || !b || !result) {
        set_msg(err, errlen, "xcal_residual_noalloc: null device pointer");
        return XCAL_ERR_INVALID;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
        set_msg(err, errlen, "xcal_residual_noalloc: no current CUDA device");
        return XCAL_ERR_CUDA;
    }
    void* scratch = nullptr;
    {
        // first call on this device: resolve the device address of the array
        // (host code must not use the symbol itself as a pointer)
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                set_msg(err, errlen, cudaGetErrorString(e));
                return XCAL_ERR_CUDA;
            }
            g_noalloc_ptr[dev] = p;
        }
        scratch = g_noalloc_ptr[dev];
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // the last-block counter must start at zero
    cudaError_t e = cudaMemsetAsync(scratch, 0, NOALLOC_HDR, s);
    if (e == cudaSuccess) {
        int tiles = (n + RED_TILE - 1) / RED_TILE;
        k_residual_noalloc<<<tiles, RED_THREADS, 0, s>>>(n, rowptr, colval, nzval, x, b,
                                                         static_cast<unsigned char*>(scratch), result);
        g_launch_count.fetch_add(1, std::memory_order_relaxed);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_msg(err, errlen, cudaGetErrorString(e));
        return XCAL_ERR_CUDA;
    }
    return XCAL_OK;
}
