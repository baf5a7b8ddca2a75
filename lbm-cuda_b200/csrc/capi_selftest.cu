// lbm_selftest_wait_timeout: drives the give-up path of the bounded mbarrier
// waits (mbar_wait_bounded) on the GPU without a fault.  The production kernels
// take that path only when a TMA copy never completes; here a CTA waits on a
// barrier that nothing arrives on and no copy targets, with a short limit, so
// the wait must run out, report through the device error word and let the
// kernel return normally.
#include "common.cuh"
#include "host.h"

namespace lbm {

int *device_error_word();

namespace {

__global__ void wait_timeout_kernel(long long limit, int arrive, int *err, long long *d_cycles)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0)
        return;
    mbar_init(&bar, 1);
    mbar_fence_init();
    if (arrive)
        mbar_arrive(&bar); // completes phase 0
    const long long t0 = clock64();
    const bool ok = mbar_wait_bounded(&bar, 0, limit);
    const long long dt = clock64() - t0;
    if (!ok && err)
        atomicOr(err, 1);
    if (d_cycles)
        *d_cycles = dt;
    mbar_inval(&bar);
}

} // namespace
} // namespace lbm

extern "C" int lbm_selftest_wait_timeout(long long limit_cycles, int arrive, long long *d_cycles, void *stream)
{
    using namespace lbm;
    if (limit_cycles < 1 || limit_cycles > kWaitLimitCycles || (arrive != 0 && arrive != 1))
        return LBM_ERR_ARG;
    int *err = device_error_word();
    if (!err)
        return LBM_ERR_DEVICE;
    wait_timeout_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(limit_cycles, arrive, err, d_cycles);
    return status(cudaGetLastError());
}
