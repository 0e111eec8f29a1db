// Allocation-free CFL time step: mhdgpu_calc_dt_noalloc (include/mhd_gpu.h).
//
// Some callers cannot allocate device memory at the point where they need a
// time step: a host framework whose own pool allocator has reserved the
// device's memory, or a service that fixes its memory footprint at start-up
// and forbids allocation afterwards.  This entry point needs no context and
// allocates nothing.  The caller passes the state and a 3-double output on
// the device; the per-block partial minima of the reduction live in the
// file-scope array below, which every GPU that loads this library holds until
// the process exits.
//
// Limits and sharing:
//  - at most NOALLOC_MAX_PARTIALS blocks of partials, i.e. nx*ny up to
//    NOALLOC_MAX_PARTIALS * NOALLOC_CELLS_PER_BLOCK cells (33,554,432, e.g.
//    8192 x 4096); larger grids are rejected with MHDGPU_ERR_INVALID;
//  - every call shares the array.  Each call writes every partial it reads
//    before reading it, so nothing needs clearing, but calls that overlap on
//    the GPU (on different streams, or from different host threads) race on
//    it and must be serialised by the caller;
//  - the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture begins;
//  - fmin and fmax drop NaN operands, so a NaN in the state does not make
//    the result NaN, exactly as in the context's calcDt (pointwise.cu); the
//    reference's loop returns NaN only when its very first cell is NaN.
#include <mutex>

#include "common.cuh"
#include "dtcore.cuh"

namespace {

constexpr int NOALLOC_THREADS = 256;
constexpr long NOALLOC_CELLS_PER_BLOCK = 2048;   // 8 cells per thread
constexpr int NOALLOC_MAX_PARTIALS = 16384;      // 128 KiB of scratch
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_dt_partials[NOALLOC_MAX_PARTIALS];

std::mutex g_setup_mutex;
double *g_partials_addr[NOALLOC_MAX_DEVICES] = {nullptr};

__global__ void noalloc_dt_partial(mhd::DtArgs a, long cells_per_block)
{
    const long begin = blockIdx.x * cells_per_block;
    const long end = begin + cells_per_block < a.plane ? begin + cells_per_block : a.plane;
    double mn = INFINITY;
    for (long o = begin + threadIdx.x; o < end; o += blockDim.x) mn = fmin(mn, mhd::cell_dt(a, o));
    for (int s = 16; s > 0; s >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, s));
    __shared__ double sm[NOALLOC_THREADS / 32];
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mn;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = INFINITY;
        for (int w = 0; w < NOALLOC_THREADS / 32; w++) v = fmin(v, sm[w]);
        a.part[blockIdx.x] = v;  // every partial read below is written here first
    }
}

// out[0] = dt with the reference's 2% hysteresis (timeAdvance.c:142-152);
// with hyperbolic cleaning out[1] = Ch from the last cell and out[2] = Cp
// (timeAdvance.c:107-112, divBcleaning.c:4-10), else both 0.
__global__ void noalloc_dt_final(mhd::DtArgs a, int nparts, double cfl, double dt0, int cleaning,
                                 double *out)
{
    double mn = INFINITY;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) mn = fmin(mn, a.part[i]);
    for (int s = 16; s > 0; s >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, s));
    __shared__ double sm[32];
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mn;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = INFINITY;
        for (int w = 0; w < (int)(blockDim.x / 32); w++) v = fmin(v, sm[w]);
        double dtmin = v * cfl;
        out[0] = (dt0 < 0.98 * dtmin || dt0 > 1.02 * dtmin) ? dtmin : dt0;
        double ch = 0.0, cp = 0.0;
        if (cleaning == 2) {
            double cx, cy;
            mhd::cell_speeds(a, a.plane - 1, cx, cy);
            ch = fmax(cx, cy);
            cp = sqrt(0.18 * ch);
        }
        out[1] = ch;
        out[2] = cp;
    }
}

// Device address of the scratch array on the current device, looked up once
// per device.
int partials_address(double **addr)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MHDGPU_ERR_CUDA;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return MHDGPU_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partials_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_dt_partials) != cudaSuccess || !p) return MHDGPU_ERR_CUDA;
        g_partials_addr[dev] = static_cast<double *>(p);
    }
    *addr = g_partials_addr[dev];
    return MHDGPU_OK;
}

}  // namespace

extern "C" int mhdgpu_calc_dt_noalloc(const double *d_uu, const mhdgpu_params *p, double dt0,
                                      double *d_out, void *stream)
{
    if (!d_uu || !p || !d_out || p->nx < 1 || p->ny < 1 || !(p->Lx > 0) || !(p->Ly > 0))
        return mhd_set_error(MHDGPU_ERR_INVALID);
    const long plane = p->nx * p->ny;
    const long nblocks = (plane + NOALLOC_CELLS_PER_BLOCK - 1) / NOALLOC_CELLS_PER_BLOCK;
    if (nblocks > NOALLOC_MAX_PARTIALS) return mhd_set_error(MHDGPU_ERR_INVALID);
    double *partials = nullptr;
    int rc = partials_address(&partials);
    if (rc != MHDGPU_OK) return mhd_set_error(rc);
    mhd::DtArgs a;
    a.uu = d_uu;
    a.plane = plane;
    a.ny = p->ny;
    a.gamma = p->adiabaticIdx;
    a.dx = p->boundaryTypeX == 0 ? p->Lx / (double)p->nx : p->Lx / (double)(p->nx - 1);
    a.dy = p->Ly / (double)p->ny;
    a.di = p->di;
    a.resist = p->resistivity;
    a.visc = p->viscosity;
    a.hall = p->Hall;
    a.part = partials;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    noalloc_dt_partial<<<(unsigned)nblocks, NOALLOC_THREADS, 0, s>>>(a, NOALLOC_CELLS_PER_BLOCK);
    if (cudaGetLastError() != cudaSuccess) return mhd_set_error(MHDGPU_ERR_CUDA);
    noalloc_dt_final<<<1, 1024, 0, s>>>(a, (int)nblocks, p->cfl, dt0, p->divBcleaning, d_out);
    if (cudaGetLastError() != cudaSuccess) return mhd_set_error(MHDGPU_ERR_CUDA);
    return MHDGPU_OK;
}
