// diag.cu -- a device check of the bounded waits the persistent kernels use.
//
// Every spin-wait in this library (the grid barrier of the persistent CG
// kernels) gives up after a bounded number of polls, sets an error flag and
// returns, so a block that never arrives ends in an error status the host
// reads (XCAL_ERR_TIMEOUT) instead of a hung GPU.  xcal_check_bounded_wait
// exercises exactly that path without any fault: one block waits at the
// barrier for a second block that is never launched, with a short poll
// limit, and reports that it gave up and that the context still runs work.
#include "case.hpp"
#include "dev_common.cuh"
#include "krylov_bodies.cuh"

namespace xcal {

// one block, waiting for a second arrival that nothing makes
__global__ void k_wait_check(unsigned int* count, int* err, long spin_limit, int* out) {
    __shared__ int sh_err;
    unsigned int nb = 0;
    const bool ok = grid_barrier(count, 2, nb, err, &sh_err, spin_limit);
    if (threadIdx.x == 0) {
        out[0] = ok ? 0 : 1;
        out[1] = *(volatile int*)err;
    }
}

__global__ void k_wait_check_after(int* out) {
    if (threadIdx.x == 0) out[2] = 42;
}

}  // namespace xcal

using namespace xcal;

extern "C" int32_t xcal_check_bounded_wait(xcal_ctx* ctx, int64_t spin_limit, int32_t* gave_up, int32_t* flag_set,
                                           int32_t* ran_after) {
    if (!ctx || spin_limit < 1 || spin_limit > BAR_SPIN_LIMIT) return XCAL_ERR_INVALID;
    try {
        XCAL_CUDA(cudaSetDevice(ctx->device));
        DBuf<unsigned int> count;
        DBuf<int> err, out;
        count.alloc(2);
        err.alloc(1);
        out.alloc(4);
        XCAL_CUDA(cudaMemset(count.p, 0, 2 * sizeof(unsigned int)));
        XCAL_CUDA(cudaMemset(err.p, 0, sizeof(int)));
        XCAL_CUDA(cudaMemset(out.p, 0, 4 * sizeof(int)));
        k_wait_check<<<1, 32>>>(count.p, err.p, (long)spin_limit, out.p);
        XCAL_CHECK_LAUNCH();
        k_wait_check_after<<<1, 32>>>(out.p);
        XCAL_CHECK_LAUNCH();
        XCAL_CUDA(cudaDeviceSynchronize());
        int h[4] = {0, 0, 0, 0};
        XCAL_CUDA(cudaMemcpy(h, out.p, sizeof(h), cudaMemcpyDeviceToHost));
        if (gave_up) *gave_up = h[0];
        if (flag_set) *flag_set = h[1];
        if (ran_after) *ran_after = h[2] == 42 ? 1 : 0;
        return XCAL_OK;
    } catch (const Error& e) {
        ctx->set_error(e.msg);
        return e.code;
    }
}
