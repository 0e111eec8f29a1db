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
//  - at most NOALLOC_MAX_BLOCKS blocks of partials, i.e. nx*ny up to
//    NOALLOC_MAX_BLOCKS * NOALLOC_CELLS_PER_BLOCK cells (33,554,432, e.g.
//    8192 x 4096); larger grids are rejected with MHDGPU_ERR_INVALID;
//  - every call shares the array.  Each call writes every partial it reads
//    before reading it, so nothing needs clearing, but calls that overlap on
//    the GPU (on different streams, or from different host threads) race on
//    it and must be serialised by the caller;
//  - the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture begins;
//  - NaN handling is the reference's, as in the context's calcDt
//    (pointwise.cu, dtcore.cuh): its MAX/MIN macros per cell, a later cell
//    whose step is NaN skipped, a NaN step of the first cell returned.
#include <mutex>

#include "common.cuh"
#include "dtcore.cuh"

namespace {

constexpr int NOALLOC_THREADS = 256;
constexpr long NOALLOC_CELLS_PER_BLOCK = 8192;   // 32 cells per thread
constexpr int NOALLOC_MAX_BLOCKS = 4096;         // 3 doubles each: 96 KiB of scratch
constexpr int NOALLOC_MAX_PARTIALS = 3 * NOALLOC_MAX_BLOCKS;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_dt_partials[NOALLOC_MAX_PARTIALS];

std::mutex g_setup_mutex;
double *g_partials_addr[NOALLOC_MAX_DEVICES] = {nullptr};

// per block: the (minimum, last negative cell, NaN flag) fold of the
// reference's running minimum (dtcore.cuh) at part[3 b ..]
__global__ void noalloc_dt_partial(mhd::DtArgs a, long cells_per_block)
{
    const long begin = blockIdx.x * cells_per_block;
    const long end = begin + cells_per_block < a.plane ? begin + cells_per_block : a.plane;
    mhd::DtFold f{INFINITY, -1.0, 0.0};
    for (long o = begin + threadIdx.x; o < end; o += blockDim.x) mhd::dt_cell_fold(a, o, f);
    for (int s = 16; s > 0; s >>= 1) {
        f.mn = fmin(f.mn, __shfl_xor_sync(0xffffffffu, f.mn, s));
        f.lastneg = fmax(f.lastneg, __shfl_xor_sync(0xffffffffu, f.lastneg, s));
        f.nanflag = fmax(f.nanflag, __shfl_xor_sync(0xffffffffu, f.nanflag, s));
    }
    __shared__ double sm[3][NOALLOC_THREADS / 32];
    if ((threadIdx.x & 31) == 0) {
        sm[0][threadIdx.x >> 5] = f.mn;
        sm[1][threadIdx.x >> 5] = f.lastneg;
        sm[2][threadIdx.x >> 5] = f.nanflag;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = INFINITY, l = -1.0, n = 0.0;
        for (int w = 0; w < NOALLOC_THREADS / 32; w++) {
            m = fmin(m, sm[0][w]);
            l = fmax(l, sm[1][w]);
            n = fmax(n, sm[2][w]);
        }
        // every partial read below is written here first
        a.part[3 * blockIdx.x] = m;
        a.part[3 * blockIdx.x + 1] = l;
        a.part[3 * blockIdx.x + 2] = n;
    }
}

// out[0] = dt with the reference's 2% hysteresis (timeAdvance.c:142-152);
// with hyperbolic cleaning out[1] = Ch from the last cell and out[2] = Cp
// (timeAdvance.c:107-112, divBcleaning.c:4-10), else both 0.
__global__ void __launch_bounds__(256) noalloc_dt_final(mhd::DtArgs a, int nblocks, double cfl, double dt0, int cleaning,
                                 double *out)
{
    double mn = INFINITY, l = -1.0, n = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
        mn = fmin(mn, a.part[3 * i]);
        l = fmax(l, a.part[3 * i + 1]);
        n = fmax(n, a.part[3 * i + 2]);
    }
    for (int s = 16; s > 0; s >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, s));
        l = fmax(l, __shfl_xor_sync(0xffffffffu, l, s));
        n = fmax(n, __shfl_xor_sync(0xffffffffu, n, s));
    }
    __shared__ double sm[3][32];
    if ((threadIdx.x & 31) == 0) {
        sm[0][threadIdx.x >> 5] = mn;
        sm[1][threadIdx.x >> 5] = l;
        sm[2][threadIdx.x >> 5] = n;
    }
    __syncthreads();
    mn = INFINITY, l = -1.0, n = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); w++) {
        mn = fmin(mn, sm[0][w]);
        l = fmax(l, sm[1][w]);
        n = fmax(n, sm[2][w]);
    }
    __shared__ double red[32];
    const double dmin = mhd::dt_resolve(a, mn, l, n, red);
    if (threadIdx.x == 0) {
        double dtmin = dmin * cfl;
        out[0] = (dt0 < 0.98 * dtmin || dt0 > 1.02 * dtmin) ? dtmin : dt0;
        double ch = 0.0, cp = 0.0;
        if (cleaning == 2) {
            double cx, cy;
            mhd::cell_speeds(a, a.plane - 1, cx, cy);
            ch = mhd::ref_max(cx, cy);
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
    if (nblocks > NOALLOC_MAX_BLOCKS) return mhd_set_error(MHDGPU_ERR_INVALID);
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
    noalloc_dt_final<<<1, 256, 0, s>>>(a, (int)nblocks, p->cfl, dt0, p->divBcleaning, d_out);
    if (cudaGetLastError() != cudaSuccess) return mhd_set_error(MHDGPU_ERR_CUDA);
    return MHDGPU_OK;
}
