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
// are served from L2; the updated state is written by step 2 and read back
// (again from L2) and overwritten by step 3.  One padded FFT row per CTA row
// and at most 128 registers per thread keep two CTAs on each SM.
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
    // shared memory: one padded FFT row per row of the CTA (68 KB for any
    // row length), so that two CTAs share an SM
    static constexpr size_t SMEM = sizeof(double2) * ROWS * NP;
};

// Load fields fa and fb (fb < 0: zero) of this group's row into the FFT row
// as fa + i fb; each thread its own 16 points, coalesced across the group.
template <int L>
__device__ __forceinline__ void yr_load(double2 *A, const double *ra, const double *rb, int j,
                                        bool valid)
{
    using G = YRGeom<L>;
    double va[16], vb[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const int i = j + m * G::T;
        va[m] = valid ? ra[i] : 0.0;
        vb[m] = (valid && rb) ? rb[i] : 0.0;
    }
#pragma unroll
    for (int m = 0; m < 16; m++) A[fpad(j + m * G::T)] = make_double2(va[m], vb[m]);
}

// One spectral operator on the row in A (natural order, already loaded):
// forward FFT, multiply by the symbol s, inverse FFT, real part to oa and
// imaginary part to ob (null: skipped).  Ends with the block synchronised.
template <int L>
__device__ __forceinline__ void yr_op(const YRArgs &a, double2 *A, int j, bool valid,
                                      const double2 *s, double *oa, double *ob)
{
    using G = YRGeom<L>;
    __syncthreads();  // the row is complete
    fft_row<L, -1>(A, a.tw, j);
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const int i = j + m * G::T;
        A[fpad(i)] = cm(A[fpad(i)], __ldg(s + i));
    }
    __syncthreads();
    fft_row<L, +1>(A, a.tw, j);
    if (valid) {
#pragma unroll
        for (int m = 0; m < 16; m++) {
            const int i = j + m * G::T;
            double2 z = A[fpad(i)];
            if (oa) oa[i] = z.x;
            if (ob) ob[i] = z.y;
        }
    }
    __syncthreads();  // A may be refilled
}

template <int L>
__global__ void __launch_bounds__(YR_THREADS, 2) yrow_kernel(YRArgs a)
{
    using G = YRGeom<L>;
    extern __shared__ __align__(128) unsigned char yr_raw[];
    double2 *Abase = reinterpret_cast<double2 *>(yr_raw);
    const int g = threadIdx.x / G::T, j = threadIdx.x % G::T;
    const long row = (long)blockIdx.x * G::ROWS + g;
    const bool valid = row < a.nx;
    double2 *A = Abase + (size_t)g * G::NP;
    const size_t plane = (size_t)a.nx * a.ny;
    const size_t ro = valid ? (size_t)row * a.ny : 0;
    // row `ro` of field v of array base (null base: null)
    auto f = [&](double *base, int v) -> double * {
        return base ? base + (size_t)v * plane + ro : nullptr;
    };
    auto fc = [&](const double *base, int v) -> const double * {
        return base ? base + (size_t)v * plane + ro : nullptr;
    };

    // ---- 1. y-derivatives: pairs (ux,uy) (rho,p) (uz,Bz) (Bx,By) [psi],
    // d/dy of every field, d2/dy2 of u and B (a second forward FFT of the
    // pair, reloaded from L2, instead of keeping the spectrum)
    const int npair = a.nvar == 9 ? 5 : 4;
    for (int q = 0; q < npair; q++) {
        const int fa = q == 0 ? UX : q == 1 ? RHO : q == 2 ? UZ : q == 3 ? BX : PSI;
        const int fb = q == 0 ? UY : q == 1 ? P : q == 2 ? BZ : q == 3 ? BY : -1;
        yr_load<L>(A, fc(a.uu, fa), fb >= 0 ? fc(a.uu, fb) : nullptr, j, valid);
        yr_op<L>(a, A, j, valid, a.s1, f(a.dudy, fa), fb >= 0 ? f(a.dudy, fb) : nullptr);
        double *o2a = nullptr, *o2b = nullptr;
        if (fa == UX && a.d2u) { o2a = f(a.d2udy2, 0); o2b = f(a.d2udy2, 1); }
        if (fa == UZ) {
            o2a = a.d2u ? f(a.d2udy2, 2) : nullptr;
            o2b = a.d2b ? f(a.d2Bdy2, 2) : nullptr;
        }
        if (fa == BX && a.d2b) { o2a = f(a.d2Bdy2, 0); o2b = f(a.d2Bdy2, 1); }
        if (o2a || o2b) {  // uniform across the block
            yr_load<L>(A, fc(a.uu, fa), fc(a.uu, fb), j, valid);
            yr_op<L>(a, A, j, valid, a.s2, o2a, o2b);
        }
    }
    {   // (Ex, Ez) = (uz By - uy Bz, uy Bx - ux By)
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
        yr_op<L>(a, A, j, valid, a.s1, f(a.dEdy, 0), f(a.dEdy, 2));
    }

    // ---- 2. right-hand side and RK3 update, point by point ------------------
    if (valid) {
        const int nv = a.nvar;
#pragma unroll 1
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
    __syncthreads();  // the updated rows are visible to the whole block

    // ---- 3. spectral y filter of the updated fields, two at a time ----------
    const int nfp = (a.nvar + 1) / 2;
    for (int q = 0; q < nfp; q++) {
        const int v = 2 * q, w = v + 1 < a.nvar ? v + 1 : -1;
        yr_load<L>(A, fc(a.uu, v), w >= 0 ? fc(a.uu, w) : nullptr, j, valid);
        yr_op<L>(a, A, j, valid, a.sf, f(a.uu, v), w >= 0 ? f(a.uu, w) : nullptr);
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
