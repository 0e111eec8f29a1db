// Self-test of the failure path of the kernels' bounded waits: a wait on an
// mbarrier that nothing completes runs out after a short limit, raises the
// context's status flag and returns, and the host reads MHDGPU_ERR_TIMEOUT
// while the context stays usable.  No fault, trap or endless loop is
// involved: the same bounded-wait helper guards every TMA wait of the x
// kernels.
#include "common.cuh"
#include "xcore.cuh"

namespace mhd {

__global__ void wait_timeout_kernel(int *flag, long long limit)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);  // one arrival expected, none made
    __syncthreads();
    mbar_wait_bounded(&bar, 0, flag, limit);
}

}  // namespace mhd

// status of a context's kernels since the last check (api.cu)
int mhd_check_flag(mhd::Ctx *c);

extern "C" int mhdgpu_selftest_wait(mhdgpu_ctx *h, double milliseconds)
{
    mhd::Ctx *c = reinterpret_cast<mhd::Ctx *>(h);
    if (!c || !(milliseconds > 0.0) || milliseconds > 2000.0) return mhd_set_error(MHDGPU_ERR_INVALID);
    MHD_CUDA_TRY(cudaSetDevice(c->device));
    int clock_khz = 0;
    MHD_CUDA_TRY(cudaDeviceGetAttribute(&clock_khz, cudaDevAttrClockRate, c->device));
    const long long limit = (long long)(milliseconds * (double)clock_khz);
    mhd::wait_timeout_kernel<<<1, 32, 0, c->stream>>>(c->dflag, limit);
    MHD_CHECK_LAUNCH();
    return mhd_check_flag(c);
}
