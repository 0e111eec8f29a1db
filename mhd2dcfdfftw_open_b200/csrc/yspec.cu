// y-direction spectral operators: derivY (calcDerivs.c:75-109), derivYY
// (calcDerivs.c:114-150) and the spectral filter filteringY (filtering.c:40-94,
// filtY from initialize.c:161-177), which the reference runs as one FFTW
// r2c -> multiply -> c2r round trip per (field, x-row).
//
// B200 design.  y is contiguous, so a CTA owns whole rows.  Two real rows a, b
// (paired as launch_yspec says) are packed as one complex row z = a + i b and
// transformed by a complex FFT
// of length ny held in shared memory (radix-4 Stockham passes, one radix-2
// pass when log2 ny is odd).  Every operator here is real (its symbol s obeys
// s(-k) = conj s(k)), so multiplying Z[k] by s over the full signed spectrum
// and transforming back gives s*a + i s*b: the real and imaginary parts are
// the two results and no spectrum has to be separated.  The reference's
// Nyquist conventions carry over: FFTW's c2r ignores the imaginary part of
// the Nyquist bin, which makes the first derivative's Nyquist term vanish
// (symbol 0 there), while the second derivative and the filter keep it.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace mhd {

constexpr int YT = 256;

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// In-place complex FFT of length N = 2^logN in shared memory, natural order
// in and out.  sign -1: forward (exp(-i...)), +1: inverse, both unnormalised.
// tw[m] = exp(-2 pi i m / N).  Called by all threads of the block.
__device__ void fft_smem(double2 *z, int N, int logN, const double2 *__restrict__ tw,
                         int sign, int tid, int nthr)
{
    int Ns = 1;
    int passes4 = logN / 2;
    const int N4 = N >> 2;
    for (int p = 0; p < passes4; p++) {
        // each thread handles butterflies t = tid, tid+nthr, ... (< N/4);
        // stage all inputs in registers before any write
        const int nb = (N4 + nthr - 1) / nthr;
        double2 o[4][8];  // up to 8 butterflies per thread (N <= 8192 at 256 threads)
        for (int b = 0; b < nb; b++) {
            int t = tid + b * nthr;
            if (t >= N4) break;
            int k = t & (Ns - 1);
            double2 v0 = z[t], v1 = z[t + N4], v2 = z[t + 2 * N4], v3 = z[t + 3 * N4];
            if (Ns > 1) {
                int step = N / (Ns * 4);
                double2 w1 = tw[k * step], w2 = tw[2 * k * step], w3 = tw[3 * k * step];
                if (sign > 0) { w1.y = -w1.y; w2.y = -w2.y; w3.y = -w3.y; }
                v1 = cmul(v1, w1);
                v2 = cmul(v2, w2);
                v3 = cmul(v3, w3);
            }
            double2 a0 = make_double2(v0.x + v2.x, v0.y + v2.y);
            double2 a1 = make_double2(v0.x - v2.x, v0.y - v2.y);
            double2 a2 = make_double2(v1.x + v3.x, v1.y + v3.y);
            double2 d = make_double2(v1.x - v3.x, v1.y - v3.y);
            // (v1 - v3) * (-i) forward, * (+i) inverse
            double2 a3 = sign < 0 ? make_double2(d.y, -d.x) : make_double2(-d.y, d.x);
            o[0][b] = make_double2(a0.x + a2.x, a0.y + a2.y);
            o[1][b] = make_double2(a1.x + a3.x, a1.y + a3.y);
            o[2][b] = make_double2(a0.x - a2.x, a0.y - a2.y);
            o[3][b] = make_double2(a1.x - a3.x, a1.y - a3.y);
        }
        __syncthreads();
        for (int b = 0; b < nb; b++) {
            int t = tid + b * nthr;
            if (t >= N4) break;
            int k = t & (Ns - 1);
            int base = (t - k) * 4 + k;
            z[base] = o[0][b];
            z[base + Ns] = o[1][b];
            z[base + 2 * Ns] = o[2][b];
            z[base + 3 * Ns] = o[3][b];
        }
        __syncthreads();
        Ns *= 4;
    }
    if (logN & 1) {  // final radix-2 pass, Ns = N/2
        const int N2 = N >> 1;
        const int nb = (N2 + nthr - 1) / nthr;
        double2 o0[16], o1[16];
        for (int b = 0; b < nb; b++) {
            int t = tid + b * nthr;
            if (t >= N2) break;
            double2 v0 = z[t], v1 = z[t + N2];
            double2 w = tw[t];
            if (sign > 0) w.y = -w.y;
            v1 = cmul(v1, w);
            o0[b] = make_double2(v0.x + v1.x, v0.y + v1.y);
            o1[b] = make_double2(v0.x - v1.x, v0.y - v1.y);
        }
        __syncthreads();
        for (int b = 0; b < nb; b++) {
            int t = tid + b * nthr;
            if (t >= N2) break;
            z[t] = o0[b];
            z[t + N2] = o1[b];
        }
        __syncthreads();
    }
}

struct YArgs {
    const double *in;
    double *out;
    const double2 *tw;
    const double2 *sym;   // complex symbol per k (k < ny, signed wavenumbers)
    long nx, ny;
    int logN;
    int nv;
    int in_start, out_start;
    int pa[5], pb[5];  // the fields of each pair (pb < 0: none)
};

// One (x-row, field pair) per CTA: out[v] = op(in[in_start + v]) for the two
// fields v = pa[pair], pb[pair] of row blockIdx.x.
__global__ void __launch_bounds__(YT) yspec_kernel(YArgs a)
{
    extern __shared__ __align__(16) double2 zsm[];
    const int N = (int)a.ny;
    const long row = blockIdx.x;
    const int v0 = a.pa[blockIdx.y];
    const int v1 = a.pb[blockIdx.y] >= 0 ? a.pb[blockIdx.y] : a.nv;  // nv: none
    const size_t plane = (size_t)a.nx * a.ny;
    const double *ra = a.in + (size_t)(a.in_start + v0) * plane + row * a.ny;
    const double *rb = v1 < a.nv ? a.in + (size_t)(a.in_start + v1) * plane + row * a.ny : nullptr;
    for (int j = threadIdx.x; j < N; j += blockDim.x)
        zsm[j] = make_double2(ra[j], rb ? rb[j] : 0.0);
    __syncthreads();
    fft_smem(zsm, N, a.logN, a.tw, -1, threadIdx.x, blockDim.x);
    for (int k = threadIdx.x; k < N; k += blockDim.x) zsm[k] = cmul(zsm[k], a.sym[k]);
    __syncthreads();
    fft_smem(zsm, N, a.logN, a.tw, +1, threadIdx.x, blockDim.x);
    double *oa = a.out + (size_t)(a.out_start + v0) * plane + row * a.ny;
    double *ob = v1 < a.nv ? a.out + (size_t)(a.out_start + v1) * plane + row * a.ny : nullptr;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        double2 z = zsm[j];
        oa[j] = z.x;
        if (ob) ob[j] = z.y;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static const double PI_REF = 3.14159265358979323846;  // acos(-1), parameter.h:14

int yspec_setup(Ctx *c)
{
    const long N = c->ny;
    const double Ly = c->p.Ly;
    const double PI = std::acos(-1.0);
    (void)PI_REF;
    std::vector<double2> tw(N), s1(N), s2(N), sf(N);
    for (long m = 0; m < N; m++) {
        long double ang = -6.283185307179586476925286766559L * (long double)m / (long double)N;
        tw[m] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
    // spectral filter filtY (initialize.c:161-177), afy = 0.45 (initialize.c:44)
    const double afy = 0.45;
    const double aj = (5.0 + 6.0 * afy) / 8.0;
    const double bj = (1.0 + 2.0 * afy) / 2.0;
    const double cj = -(1.0 - 2 * afy) / 8.0;
    for (long k = 0; k < N; k++) {
        long kk = k <= N / 2 ? k : N - k;  // |signed wavenumber|
        double sgn = k <= N / 2 ? 1.0 : -1.0;
        // derivY: i * 2 pi / Ly * k / ny; zero at Nyquist (c2r drops it)
        double f1 = 2 * PI / Ly * (double)kk / (double)N;
        s1[k] = make_double2(0.0, (k == N / 2) ? 0.0 : sgn * f1);
        // derivYY: -(2 pi / Ly * k)^2 / ny, Nyquist kept
        double q = 2 * PI / Ly * (double)kk;
        s2[k] = make_double2(-(q * q) / (double)N, 0.0);
        double w = 2. * PI * (double)kk / (double)N;
        double filt = (aj + bj * std::cos(w) + cj * std::cos(2 * w)) / (1 + 2 * afy * std::cos(w));
        sf[k] = make_double2(filt / (double)N, 0.0);
    }
    MHD_CUDA_TRY(cudaMalloc(&c->tw, sizeof(double2) * N));
    double2 *sym;
    MHD_CUDA_TRY(cudaMalloc(&sym, sizeof(double2) * N * 3));
    MHD_CUDA_TRY(cudaMemcpy(c->tw, tw.data(), sizeof(double2) * N, cudaMemcpyHostToDevice));
    MHD_CUDA_TRY(cudaMemcpy(sym, s1.data(), sizeof(double2) * N, cudaMemcpyHostToDevice));
    MHD_CUDA_TRY(cudaMemcpy(sym + N, s2.data(), sizeof(double2) * N, cudaMemcpyHostToDevice));
    MHD_CUDA_TRY(cudaMemcpy(sym + 2 * N, sf.data(), sizeof(double2) * N, cudaMemcpyHostToDevice));
    c->ysym_d1 = reinterpret_cast<double *>(sym);
    c->ysym_d2 = reinterpret_cast<double *>(sym + N);
    c->ysym_f = reinterpret_cast<double *>(sym + 2 * N);
    // FP32 tables: twiddles, the two derivative symbols, and the filter
    // symbol minus the identity (1/N with the unnormalised transforms)
    std::vector<float2> t32(4 * N);
    for (long k = 0; k < N; k++) {
        t32[k] = make_float2((float)tw[k].x, (float)tw[k].y);
        t32[N + k] = make_float2((float)s1[k].x, (float)s1[k].y);
        t32[2 * N + k] = make_float2((float)s2[k].x, (float)s2[k].y);
        t32[3 * N + k] = make_float2((float)(sf[k].x - 1.0 / (double)N), (float)sf[k].y);
    }
    MHD_CUDA_TRY(cudaMalloc(&c->ytab32, sizeof(float2) * 4 * N));
    MHD_CUDA_TRY(cudaMemcpy(c->ytab32, t32.data(), sizeof(float2) * 4 * N, cudaMemcpyHostToDevice));
    MHD_CUDA_TRY(cudaFuncSetAttribute(yspec_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(sizeof(double2) * 8192)));
    return MHDGPU_OK;
}

void yspec_free(Ctx *c)
{
    cudaFree(c->tw);
    cudaFree(c->ysym_d1);
    cudaFree(c->ytab32);
    c->ytab32 = nullptr;
    c->tw = nullptr;
    c->ysym_d1 = c->ysym_d2 = c->ysym_f = nullptr;
}

// op: 0 first derivative, 1 second derivative, 2 spectral filter
int launch_yspec(Ctx *c, int op, int nv, const double *in, int in_start, double *out,
                 int out_start)
{
    if (nv <= 0) return MHDGPU_OK;
    YArgs a;
    a.in = in;
    a.out = out;
    a.tw = c->tw;
    a.sym = reinterpret_cast<const double2 *>(op == 0 ? c->ysym_d1 : op == 1 ? c->ysym_d2 : c->ysym_f);
    a.nx = c->nx;
    a.ny = c->ny;
    int logN = 0;
    while ((1L << logN) < c->ny) logN++;
    a.logN = logN;
    a.nv = nv;
    a.in_start = in_start;
    a.out_start = out_start;
    // Which fields share a complex transform.  A whole state (8 or 9 fields
    // from field 0) is paired (ux, uy) (rho, p) (uz, Bz) (Bx, By) [psi], so
    // that the out-of-plane family never shares a transform with an in-plane
    // field and a field the reference keeps exactly zero (uz, Bz of a 2-D
    // flow) stays exactly zero; 3-field sets (u, B, E) pair (x, y) and leave
    // z alone; other sets pair consecutive fields.
    int np = 0;
    if (nv >= 8 && nv <= 9 && in_start == 0 && out_start == 0) {
        const int pa[5] = {UX, RHO, UZ, BX, PSI}, pb[5] = {UY, P, BZ, BY, -1};
        np = nv == 9 ? 5 : 4;
        for (int q = 0; q < np; q++) {
            a.pa[q] = pa[q];
            a.pb[q] = pb[q];
        }
    } else {
        if (nv > 10) return mhd_set_error(MHDGPU_ERR_INVALID);
        for (int v = 0; v < nv; v += 2, np++) {
            a.pa[np] = v;
            a.pb[np] = v + 1 < nv ? v + 1 : -1;
        }
    }
    dim3 grid((unsigned)c->nx, (unsigned)np, 1);
    int thr = (int)std::min<long>(YT, std::max<long>(32, c->ny / 4));
    prof_begin(c, KC_YSPEC, (double)c->nx * c->ny * 8.0 * 2.0 * nv);
    yspec_kernel<<<grid, thr, sizeof(double2) * c->ny, c->stream>>>(a);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    return MHDGPU_OK;
}

}  // namespace mhd
