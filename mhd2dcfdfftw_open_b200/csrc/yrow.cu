// y pass of the fused RK3 stage (see fused.cu), one kernel per stage.  For
// each x-row (y contiguous), in shared memory and registers:
//   1. the y-derivatives of the stage (derivY / derivYY, calcDerivs.c:75-150):
//      two real fields packed as one complex row, one forward FFT, then per
//      operator a symbol multiply and one inverse FFT -- d/dy of all fields,
//      d2/dy2 of u and B, d/dy of Ex and Ez (E = -u x B, calcRHS.c:24-43,
//      formed while the row is loaded);
//   2. calcRHS (calcRHS.c:46-75, 498-544) and rkExecute (timeAdvance.c:29-36)
//      point by point;
//   3. the spectral y filter (filteringY, filtering.c:40-94) of the updated
//      fields.
// The derivative rows pass through the context's dudy/d2udy2/d2Bdy2/dEdy
// arrays, written in step 1 and read back in step 2 by the same CTA, so they
// are served from L2; the updated state is written once by step 2 and the
// filtered state once by step 3.
#include "common.cuh"
#include "fft.cuh"
#include "rhscore.cuh"
#include "xcore.cuh"

namespace mhd {

constexpr int YR_THREADS = 256;

struct YRArgs {
    double *uu, *dudtRK;
    const double *dudx, *d2udx2, *d2Bdx2, *dEdx;
    double *dudy, *d2udy2, *d2Bdy2, *dEdy;
    const double2 *tw, *s1, *s2, *sf;  // twiddles; symbols of d/dy, d2/dy2, filter
    long nx, ny;
    int nvar;
    RhsCoef k;
    double cc, dd;
    int read_rk, write_rk;
    int d2u, d2b;  // second derivatives of u (viscosity) and B (resistivity or Hall)
    int *flag;     // status flag of bounded waits
};

template <int L>
struct YRGeom {
    static constexpr int N = 1 << L;
    static constexpr int T = N / 16;                                  // threads per row
    static constexpr int ROWS = T >= YR_THREADS ? 1 : YR_THREADS / T;  // rows per CTA
    static constexpr int NP = N + N / 16;                             // padded row
    // shared memory: FFT rows (ROWS x NP double2), staging of two raw rows
    // per row (ROWS x 2N double), one mbarrier
    static constexpr size_t SMEM = sizeof(double2) * ROWS * NP + sizeof(double) * ROWS * 2 * N + 16;
};

// TMA bulk copies of state fields fa and fb (fb < 0: none) of the block's rows
// into the staging buffer; called by warp 0.  Completion is counted on `bar`.
template <int L>
__device__ __forceinline__ void yr_prefetch(const YRArgs &a, double *S, uint64_t *bar, long row0,
                                            int fa, int fb)
{
    using G = YRGeom<L>;
    const size_t plane = (size_t)a.nx * a.ny;
    const int nrows = (int)min((long)G::ROWS, a.nx - row0);
    const unsigned rowb = (unsigned)G::N * 8u;
    if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(bar, rowb * (unsigned)nrows * (fb >= 0 ? 2u : 1u));
    }
    __syncwarp();
    for (int q = threadIdx.x; q < 2 * nrows; q += 32) {
        const int g = q >> 1, which = q & 1;
        const int fld = which ? fb : fa;
        if (fld < 0) continue;
        bulk_g2s(S + (size_t)g * 2 * G::N + (size_t)which * G::N,
                 a.uu + (size_t)fld * plane + (size_t)(row0 + g) * a.ny, rowb, bar);
    }
}

// Spectral operators of one pair: A holds the row packed as re + i im.
// Forward FFT, then for each of up to two symbols: multiply, inverse FFT,
// write the real part to oa and the imaginary part to ob (null: skipped).
// The spectrum is kept in registers between the two operators.
template <int L>
__device__ void yr_ops(const YRArgs &a, double2 *A, int j, bool valid, long row,
                       const double2 *sA, double *oA1, double *oB1, const double2 *sB, double *oA2,
                       double *oB2)
{
    using G = YRGeom<L>;
    const size_t ro = (size_t)row * a.ny;
    fft_row<L, -1>(A, a.tw, j);
    double2 Z[16];
#pragma unroll
    for (int m = 0; m < 16; m++) Z[m] = A[fpad(j + m * G::T)];
    for (int op = 0; op < 2; op++) {
        const double2 *s = op == 0 ? sA : sB;
        double *oa = op == 0 ? oA1 : oA2, *ob = op == 0 ? oB1 : oB2;
        if (!s) continue;  // uniform across the block
        if (op == 1) __syncthreads();  // previous inverse FFT's results are stored
#pragma unroll
        for (int m = 0; m < 16; m++) {
            const int i = j + m * G::T;
            A[fpad(i)] = cm(Z[m], __ldg(s + i));
        }
        __syncthreads();
        fft_row<L, +1>(A, a.tw, j);
        if (valid) {
#pragma unroll
            for (int m = 0; m < 16; m++) {
                const int i = j + m * G::T;
                double2 z = A[fpad(i)];
                if (oa) oa[ro + i] = z.x;
                if (ob) ob[ro + i] = z.y;
            }
        }
    }
    __syncthreads();
}

// Unpack the staged raw rows of this group into the FFT row.
template <int L>
__device__ __forceinline__ void yr_unpack(double2 *A, const double *Sg, int j, bool two)
{
    using G = YRGeom<L>;
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const int i = j + m * G::T;
        A[fpad(i)] = make_double2(Sg[i], two ? Sg[G::N + i] : 0.0);
    }
}

template <int L>
__global__ void __launch_bounds__(YR_THREADS, 1) yrow_kernel(YRArgs a)
{
    using G = YRGeom<L>;
    extern __shared__ __align__(128) unsigned char yr_raw[];
    double2 *Abase = reinterpret_cast<double2 *>(yr_raw);
    double *S = reinterpret_cast<double *>(Abase + (size_t)G::ROWS * G::NP);
    uint64_t *bar = reinterpret_cast<uint64_t *>(S + (size_t)G::ROWS * 2 * G::N);
    const int g = threadIdx.x / G::T, j = threadIdx.x % G::T;
    const long row0 = (long)blockIdx.x * G::ROWS;
    const long row = row0 + g;
    const bool valid = row < a.nx;
    double2 *A = Abase + (size_t)g * G::NP;
    const double *Sg = S + (size_t)g * 2 * G::N;
    const size_t plane = (size_t)a.nx * a.ny;
    auto f = [&](double *base, int v) -> double * { return base ? base + (size_t)v * plane : nullptr; };
    unsigned ph = 0;

    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();

    // ---- 1. y-derivatives; the pairs' rows are staged by TMA one pair ahead
    // (pairs: (ux,uy) (rho,p) (uz,Bz) (Bx,By) [psi]; (Ex,Ez) is formed from
    // the state with plain loads)
    const int pa[5] = {UX, RHO, UZ, BX, PSI};
    const int pb[5] = {UY, P, BZ, BY, -1};
    const int npair = a.nvar == 9 ? 5 : 4;
    if (threadIdx.x < 32) yr_prefetch<L>(a, S, bar, row0, pa[0], pb[0]);
    for (int q = 0; q < npair; q++) {
        mbar_wait_bounded(bar, ph, a.flag);
        ph ^= 1u;
        yr_unpack<L>(A, Sg, j, pb[q] >= 0);
        __syncthreads();  // staging consumed: the next pair may land in it
        if (q + 1 < npair && threadIdx.x < 32) yr_prefetch<L>(a, S, bar, row0, pa[q + 1], pb[q + 1]);
        const int fa = pa[q], fb = pb[q];
        const double2 *s2 = nullptr;
        double *o2a = nullptr, *o2b = nullptr;
        if (fa == UX && a.d2u) { s2 = a.s2; o2a = f(a.d2udy2, 0); o2b = f(a.d2udy2, 1); }
        if (fa == UZ && (a.d2u || a.d2b)) {
            s2 = a.s2;
            o2a = a.d2u ? f(a.d2udy2, 2) : nullptr;
            o2b = a.d2b ? f(a.d2Bdy2, 2) : nullptr;
        }
        if (fa == BX && a.d2b) { s2 = a.s2; o2a = f(a.d2Bdy2, 0); o2b = f(a.d2Bdy2, 1); }
        yr_ops<L>(a, A, j, valid, row, a.s1, f(a.dudy, fa), fb >= 0 ? f(a.dudy, fb) : nullptr, s2,
                  o2a, o2b);
    }
    {   // (Ex, Ez) = (uz By - uy Bz, uy Bx - ux By)
        const size_t ro = (size_t)row * a.ny;
#pragma unroll 4
        for (int m = 0; m < 16; m++) {
            const int i = j + m * G::T;
            double2 z = make_double2(0.0, 0.0);
            if (valid) {
                const double *u = a.uu + ro + i;
                double ux = u[UX * plane], uy = u[UY * plane], uz = u[UZ * plane];
                double bx = u[BX * plane], by = u[BY * plane], bz = u[BZ * plane];
                z = make_double2(uz * by - uy * bz, uy * bx - ux * by);
            }
            A[fpad(i)] = z;
        }
        __syncthreads();
        yr_ops<L>(a, A, j, valid, row, a.s1, f(a.dEdy, 0), f(a.dEdy, 2), nullptr, nullptr, nullptr);
    }

    // ---- 2. right-hand side and RK3 update, point by point ------------------
    if (valid) {
        const size_t ro = (size_t)row * a.ny;
        const int nv = a.nvar;
        for (int m = 0; m < 16; m++) {
            const size_t o = ro + j + m * G::T;
            double u[9], dx[9], dy[9], d2x[6], d2y[6], r[9];
#pragma unroll
            for (int v = 0; v < 9; v++) {
                if (v < nv) {
                    u[v] = a.uu[v * plane + o];
                    dx[v] = a.dudx[v * plane + o];
                    dy[v] = a.dudy[v * plane + o];
                } else {
                    u[v] = dx[v] = dy[v] = 0.0;
                }
            }
#pragma unroll
            for (int c = 0; c < 3; c++) {
                d2x[c] = a.k.visc > 0 ? a.d2udx2[c * plane + o] : 0.0;
                d2y[c] = a.k.visc > 0 ? a.d2udy2[c * plane + o] : 0.0;
                d2x[3 + c] = a.k.resist > 0 ? a.d2Bdx2[c * plane + o] : 0.0;
                d2y[3 + c] = a.k.resist > 0 ? a.d2Bdy2[c * plane + o] : 0.0;
            }
            rhs_point(a.k, u, dx, dy, d2x, d2y, a.dEdx[plane + o], a.dEdx[2 * plane + o],
                      a.dEdy[o], a.dEdy[2 * plane + o], 0.0, 0.0, r);
#pragma unroll
            for (int v = 0; v < 9; v++) {
                if (v < nv) {
                    double rk = a.read_rk ? a.dudtRK[v * plane + o] : 0.0;
                    a.uu[v * plane + o] = u[v] + a.cc * r[v] + a.dd * rk;
                    if (a.write_rk) a.dudtRK[v * plane + o] = r[v];
                }
            }
        }
    }
    // the updated rows are read back by the TMA (async proxy) below
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __syncthreads();

    // ---- 3. spectral y filter of the updated fields, staged one pair ahead --
    const int nfp = (a.nvar + 1) / 2;
    if (threadIdx.x < 32) yr_prefetch<L>(a, S, bar, row0, 0, 1);
    for (int q = 0; q < nfp; q++) {
        const int v = 2 * q, w = v + 1 < a.nvar ? v + 1 : -1;
        mbar_wait_bounded(bar, ph, a.flag);
        ph ^= 1u;
        yr_unpack<L>(A, Sg, j, w >= 0);
        __syncthreads();
        if (q + 1 < nfp && threadIdx.x < 32) {
            const int v2 = 2 * (q + 1), w2 = v2 + 1 < a.nvar ? v2 + 1 : -1;
            yr_prefetch<L>(a, S, bar, row0, v2, w2);
        }
        yr_ops<L>(a, A, j, valid, row, a.sf, f(a.uu, v), w >= 0 ? f(a.uu, w) : nullptr, nullptr,
                  nullptr, nullptr);
    }
}

template <int L>
static int launch_yrow_l(Ctx *c, const YRArgs &a, double bytes)
{
    using G = YRGeom<L>;
    const size_t smem = G::SMEM;
    static bool attr_done[64] = {false};  // per device
    int dev = 0;
    MHD_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
    if (!attr_done[dev]) {
        MHD_CUDA_TRY(cudaFuncSetAttribute(yrow_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        attr_done[dev] = true;
    }
    const unsigned grid = (unsigned)((c->nx + G::ROWS - 1) / G::ROWS);
    prof_begin(c, KC_FUSED_Y, bytes);
    yrow_kernel<L><<<grid, G::T * G::ROWS, smem, c->stream>>>(a);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    return MHDGPU_OK;
}

// Whether the row kernel serves this context (16 <= ny <= 4096).
bool yrow_supported(const Ctx *c) { return c->ny >= 16 && c->ny <= 4096; }

int launch_yrow(Ctx *c, int iRK, int last_stage)
{
    const mhdgpu_params &p = c->p;
    YRArgs a;
    a.uu = c->arr[MHDGPU_UU];
    a.dudtRK = c->arr[MHDGPU_DUDTRK];
    a.dudx = c->arr[MHDGPU_DUDX];
    a.d2udx2 = c->arr[MHDGPU_D2UDX2];
    a.d2Bdx2 = c->arr[MHDGPU_D2BDX2];
    a.dEdx = c->arr[MHDGPU_DEDX];
    a.dudy = c->arr[MHDGPU_DUDY];
    a.d2udy2 = c->arr[MHDGPU_D2UDY2];
    a.d2Bdy2 = c->arr[MHDGPU_D2BDY2];
    a.dEdy = c->arr[MHDGPU_DEDY];
    a.tw = c->tw;
    a.s1 = reinterpret_cast<const double2 *>(c->ysym_d1);
    a.s2 = reinterpret_cast<const double2 *>(c->ysym_d2);
    a.sf = reinterpret_cast<const double2 *>(c->ysym_f);
    a.nx = c->nx;
    a.ny = c->ny;
    a.nvar = c->nvar;
    a.k = RhsCoef{p.adiabaticIdx, p.viscosity, p.resistivity, c->const_diff_divb, c->Ch, c->Cp,
                  p.divBcleaning};
    a.cc = c->cc[iRK];
    a.dd = c->dd[iRK];
    a.read_rk = iRK > 0;       // dd[0] = 0 and dudtRK is zero at the first stage
    a.write_rk = !last_stage;  // rkInit clears dudtRK after the last stage
    a.d2u = p.viscosity > 0;
    a.d2b = p.resistivity > 0 || p.Hall == 1;
    a.flag = c->dflag;
    // algorithmic bytes: state + x derivatives + dudtRK read, state (twice:
    // update and filter) + dudtRK written
    const int nx_der = c->nvar + (a.d2u ? 3 : 0) + (a.d2b ? 3 : 0) + 2;
    const double bytes = (double)c->nx * c->ny * 8.0 *
                         (c->nvar + nx_der + (a.read_rk ? c->nvar : 0) + c->nvar +
                          (a.write_rk ? c->nvar : 0));
    switch (c->ny) {
    case 16: return launch_yrow_l<4>(c, a, bytes);
    case 32: return launch_yrow_l<5>(c, a, bytes);
    case 64: return launch_yrow_l<6>(c, a, bytes);
    case 128: return launch_yrow_l<7>(c, a, bytes);
    case 256: return launch_yrow_l<8>(c, a, bytes);
    case 512: return launch_yrow_l<9>(c, a, bytes);
    case 1024: return launch_yrow_l<10>(c, a, bytes);
    case 2048: return launch_yrow_l<11>(c, a, bytes);
    case 4096: return launch_yrow_l<12>(c, a, bytes);
    default: return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
    }
}

}  // namespace mhd
