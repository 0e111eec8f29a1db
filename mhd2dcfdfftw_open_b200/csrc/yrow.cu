// y pass of the fused RK3 stage (see fused.cu), one kernel per stage.  For
// each x-row (y contiguous), in shared memory and registers:
//   1. the y-derivatives of the stage (derivY / derivYY, calcDerivs.c:75-150):
//      two real fields packed as one complex row, one forward FFT, then per
//      operator a symbol multiply and one inverse FFT -- d/dy of all fields,
//      d2/dy2 of u and B, d/dy of Ex and Ez (E = -u x B, calcRHS.c:24-43,
//      formed while the row is loaded).  Pairs never mix the out-of-plane
//      family (uz, Bz, Ex, Ey) with an in-plane field, so fields that the
//      reference's per-field real transforms keep exactly zero stay zero;
//   2. calcRHS (calcRHS.c:46-75, 498-544) and rkExecute (timeAdvance.c:29-36)
//      point by point;
//   3. the spectral y filter (filteringY, filtering.c:40-94) of the updated
//      fields.
// The derivative rows pass through the context's dudy/d2udy2/d2Bdy2/dEdy
// arrays, written in step 1 and read back in step 2 by the same CTA, so they
// are served from L2; the updated state is written by step 2 and read back
// (again from L2) and overwritten by step 3.  One padded FFT row per CTA row
// and at most 128 registers per thread keep two CTAs on each SM.
#include <mutex>

#include "common.cuh"
#include "fft.cuh"
#include "rhscore.cuh"
#include "xcore.cuh"

namespace mhd {

constexpr int YR_THREADS = 256;

struct YRArgs {
    const double *uin;  // the state the stage starts from (uu, or the x filter's copy)
    double *uu, *dudtRK;  // the updated state is written to uu
    double *spec;  // the context's dudt array: per-row scratch of d2/dy2 spectra
    // derivative arrays: doubles, or floats (field v at v * nx * ny) in the
    // mixed-precision stage
    const void *dudx, *d2udx2, *d2Bdx2, *dEdx;
    void *dudy, *d2udy2, *d2Bdy2, *dEdy;
    const double2 *tw, *s1, *s2, *sf;  // twiddles; symbols of d/dy, d2/dy2, filter
    const float2 *tw32, *s1_32, *s2_32, *sfd32;  // float twiddles, symbols, filter - identity
    long nx, ny;
    int nvar;
    RhsCoef k;
    double cc, dd;
    // device step control: with dtdev, cc = ccoef dt and dd = dcoef dt with
    // dt = dtdev[0], and Ch, Cp = dtdev[1], dtdev[2] (hyperbolic cleaning)
    const double *dtdev;
    double ccoef, dcoef;
    // 0: the whole y pass; 1: its y derivatives only; 2: the rest (RHS,
    // RK3, filter), with d(divB)/dx, d(divB)/dy read for diffusive cleaning
    int mode;
    const double *ddivbdx, *ddivbdy;
    int read_rk, write_rk;
    int d2u, d2b;  // second derivatives of u (viscosity) and B (resistivity or Hall)
    int *flag;     // status flag of bounded waits
};

template <typename T> struct YRCplx;
template <> struct YRCplx<double> { using C = double2; };
template <> struct YRCplx<float> { using C = float2; };

template <int L, typename T>
struct YRGeom {
    using C = typename YRCplx<T>::C;
    static constexpr int N = 1 << L;
    static constexpr int T_ = N / 16;                                   // threads per row
    static constexpr int ROWS = T_ >= YR_THREADS ? 1 : YR_THREADS / T_;  // rows per CTA
    // threads per CTA: YR_THREADS, or one row of 8192 points by 512 threads
    static constexpr int THREADS = T_ * ROWS;
    static constexpr int NP = N + N / 16;                              // padded row
    // shared memory: one padded FFT row per row of the CTA (68 KB in FP64,
    // 34 KB in FP32, for rows up to 4096 points; twice that for 8192)
    static constexpr size_t SMEM = sizeof(C) * ROWS * NP;
    // CTAs per SM the register budget is set for.  Measured at 4096^2 on one
    // B200: FP64 at 2 (128 registers) 5.05 ms per launch, at 3 (80) 5.88 ms;
    // FP32 at 2 5.04 ms, 3 4.11 ms, 4 (64 registers, 136 KB of shared memory
    // per SM) 3.65 ms -- more resident rows beat fewer spills, up to where
    // the spills reach the FP64 working set
    static constexpr int MINB = THREADS > YR_THREADS ? 1 : (sizeof(T) == 8 ? 2 : 4);
};

// Load fields fa and fb (fb < 0: zero) of this group's row into the FFT row
// as (fa - ca) + i (fb - cb); each thread its own 16 points, coalesced across
// the group.  ca/cb are 0 in FP64; in FP32 they are the row's first values,
// subtracted in FP64: the operators applied here (d/dy, d2/dy2 and filter
// minus identity) map constants to zero, and the FP32 row then carries only
// the variation along the row.
template <int L, typename T>
__device__ __forceinline__ void yr_load(typename YRCplx<T>::C *A, const double *ra,
                                        const double *rb, double ca, double cb, int j, bool valid)
{
    using G = YRGeom<L, T>;
    double va[16], vb[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const int i = j + m * G::T_;
        va[m] = valid ? ra[i] : 0.0;
        vb[m] = (valid && rb) ? rb[i] : 0.0;
    }
#pragma unroll
    for (int m = 0; m < 16; m++)
        A[fpad(j + m * G::T_)] = cmk<typename G::C>((T)(va[m] - ca), (T)(vb[m] - cb));
}

// One spectral operator on the row in A (natural order, already loaded):
// forward FFT, multiply by the symbol s, inverse FFT; the real part goes to
// oa and the imaginary part to ob (null: skipped), stored as T, or with ACC
// added to the doubles there.  Ends with the block synchronised.
template <int L, typename T, bool ACC, typename O>
__device__ __forceinline__ void yr_op(const typename YRCplx<T>::C *tw, typename YRCplx<T>::C *A,
                                      int j, bool valid, const typename YRCplx<T>::C *s, O *oa,
                                      O *ob)
{
    using G = YRGeom<L, T>;
    __syncthreads();  // the row is complete
    fft_row<L, -1>(A, tw, j);
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const int i = j + m * G::T_;
        A[fpad(i)] = cm(A[fpad(i)], __ldg(s + i));
    }
    __syncthreads();
    fft_row<L, +1>(A, tw, j);
    if (valid) {
#pragma unroll
        for (int m = 0; m < 16; m++) {
            const int i = j + m * G::T_;
            const typename G::C z = A[fpad(i)];
            if constexpr (ACC) {
                if (oa) oa[i] += (double)z.x;
                if (ob) ob[i] += (double)z.y;
            } else {
                if (oa) oa[i] = (O)z.x;
                if (ob) ob[i] = (O)z.y;
            }
        }
    }
    __syncthreads();  // A may be refilled
}

// d/dy and d2/dy2 of one pair from one forward FFT: the d2/dy2 spectrum is
// parked in global scratch (element i < N/2 at lo[i], the others at hi[i];
// each thread parks and takes back its own elements, so no barrier guards
// it) while the d/dy inverse runs in A.
template <int L, typename T>
__device__ __forceinline__ void yr_op12(const typename YRCplx<T>::C *tw, typename YRCplx<T>::C *A,
                                        int j, bool valid, const typename YRCplx<T>::C *s1,
                                        const typename YRCplx<T>::C *s2,
                                        typename YRCplx<T>::C *lo, typename YRCplx<T>::C *hi,
                                        T *o1a, T *o1b, T *o2a, T *o2b)
{
    using G = YRGeom<L, T>;
    using C = typename G::C;
    __syncthreads();  // the row is complete
    fft_row<L, -1>(A, tw, j);
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const int i = j + m * G::T_;
        const C z = A[fpad(i)];
        // i < N/2 exactly when m < 8; rows past the grid park nothing
        if (valid) (m < 8 ? lo : hi)[i] = cm(z, __ldg(s2 + i));
        A[fpad(i)] = cm(z, __ldg(s1 + i));
    }
    __syncthreads();
    fft_row<L, +1>(A, tw, j);
    if (valid) {
#pragma unroll
        for (int m = 0; m < 16; m++) {
            const int i = j + m * G::T_;
            const C z = A[fpad(i)];
            if (o1a) o1a[i] = z.x;
            if (o1b) o1b[i] = z.y;
        }
    }
    __syncthreads();  // every thread has read its d/dy values
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const int i = j + m * G::T_;
        A[fpad(i)] = valid ? (m < 8 ? lo : hi)[i] : cmk<C>((T)0, (T)0);
    }
    __syncthreads();
    fft_row<L, +1>(A, tw, j);
    if (valid) {
#pragma unroll
        for (int m = 0; m < 16; m++) {
            const int i = j + m * G::T_;
            const C z = A[fpad(i)];
            if (o2a) o2a[i] = z.x;
            if (o2b) o2b[i] = z.y;
        }
    }
    __syncthreads();  // A may be refilled
}

// d/dy of one real row per half of the CTA (one CTA per row of N = 2^L
// points), each through a complex FFT of M = N/2 points: the row's even
// samples as the real part, the odd ones as the imaginary part.  The N-point
// spectrum follows from the M-point one (X_k = A_k + W^k B_k and X_{k+M} =
// A_k - W^k B_k, A and B the spectra of the even and odd samples, W =
// exp(-2 pi i / N)); it is multiplied by the d/dy symbol and folded back the
// same way for the inverse M-point FFT.  Each field is transformed alone, as
// the reference's real transforms do, so a field that is zero stays exactly
// zero.  get(g, i): sample i of the half's field g; put(g, i, v) stores the
// result.  Ends with the block synchronised.
template <int L, typename T, class Get, class Put>
__device__ __forceinline__ void yr_real_pair(typename YRCplx<T>::C *Abase,
                                             const typename YRCplx<T>::C *tw,
                                             const typename YRCplx<T>::C *s1, Get get, Put put)
{
    using C = typename YRCplx<T>::C;
    constexpr int N = 1 << L, M = N / 2, TH = M / 16;
    static_assert(TH * 2 == YRGeom<L, T>::T_, "one row per CTA, two halves");
    const int g = threadIdx.x / TH, jj = threadIdx.x % TH;
    C *Z = Abase + (size_t)g * (M + M / 16);
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const int n = jj + m * TH;
        Z[fpad(n)] = cmk<C>(get(g, 2 * n), get(g, 2 * n + 1));
    }
    __syncthreads();
    fft_row<L - 1, -1, C, 2>(Z, tw, jj);
    C zk[16], zm[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const int k = jj + m * TH;
        zk[m] = Z[fpad(k)];
        zm[m] = Z[fpad((M - k) & (M - 1))];
    }
    __syncthreads();
    using R = creal_t<C>;
    const R h = (R)0.5;
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const int k = jj + m * TH;
        const C a = cmk<C>(h * (zk[m].x + zm[m].x), h * (zk[m].y - zm[m].y));   // (Z_k + conj Z_-k)/2
        const C b = cmk<C>(h * (zk[m].y + zm[m].y), -h * (zk[m].x - zm[m].x));  // (Z_k - conj Z_-k)/(2i)
        const C w = __ldg(tw + k);
        const C wb = cm(w, b);
        const C y0 = cm(__ldg(s1 + k), ca(a, wb));
        const C y1 = cm(__ldg(s1 + k + M), cs(a, wb));
        const C e = ca(y0, y1);
        const C o = cm(cs(y0, y1), cmk<C>(w.x, -w.y));  // times exp(+2 pi i k / N)
        Z[fpad(k)] = cmk<C>(e.x - o.y, e.y + o.x);       // e + i o
    }
    __syncthreads();
    fft_row<L - 1, +1, C, 2>(Z, tw, jj);
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const int n = jj + m * TH;
        const C z = Z[fpad(n)];
        put(g, 2 * n, z.x);
        put(g, 2 * n + 1, z.y);
    }
    __syncthreads();
}

template <int L, typename T>
__global__ void __launch_bounds__((YRGeom<L, T>::THREADS), (YRGeom<L, T>::MINB)) yrow_kernel(YRArgs a)
{
    using G = YRGeom<L, T>;
    using C = typename G::C;
    constexpr bool MIX = sizeof(T) == 4;
    extern __shared__ __align__(128) unsigned char yr_raw[];
    C *Abase = reinterpret_cast<C *>(yr_raw);
    const int g = threadIdx.x / G::T_, j = threadIdx.x % G::T_;
    const long row = (long)blockIdx.x * G::ROWS + g;
    const bool valid = row < a.nx;
    C *A = Abase + (size_t)g * G::NP;
    const size_t plane = (size_t)a.nx * a.ny;
    const size_t ro = valid ? (size_t)row * a.ny : 0;
    const C *tw = MIX ? reinterpret_cast<const C *>(a.tw32) : reinterpret_cast<const C *>(a.tw);
    const C *s1 = MIX ? reinterpret_cast<const C *>(a.s1_32) : reinterpret_cast<const C *>(a.s1);
    const C *s2 = MIX ? reinterpret_cast<const C *>(a.s2_32) : reinterpret_cast<const C *>(a.s2);
    // row `ro` of field v of a derivative array of T (null base: null)
    auto f = [&](void *base, int v) -> T * {
        return base ? reinterpret_cast<T *>(base) + (size_t)v * plane + ro : nullptr;
    };
    auto fc = [&](const void *base, int v) -> const T * {
        return base ? reinterpret_cast<const T *>(base) + (size_t)v * plane + ro : nullptr;
    };
    auto su = [&](int v) -> double * { return a.uu + (size_t)v * plane + ro; };
    auto si = [&](int v) -> const double * { return a.uin + (size_t)v * plane + ro; };
    // the row shift of the FP32 operators (see yr_load)
    auto sh = [&](const double *r) -> double { return MIX && valid ? r[0] : 0.0; };

    // ---- 1. y-derivatives: pairs (ux,uy) (rho,p) (uz,Bz) (Bx,By) [psi],
    // d/dy of every field, d2/dy2 of u and B (a second forward FFT of the
    // pair, reloaded from L2, instead of keeping the spectrum)
    const int npair = a.nvar == 9 ? 5 : 4;
    for (int q = 0; q < (a.mode == 2 ? 0 : npair); q++) {
        const int fa = q == 0 ? UX : q == 1 ? RHO : q == 2 ? UZ : q == 3 ? BX : PSI;
        const int fb = q == 0 ? UY : q == 1 ? P : q == 2 ? BZ : q == 3 ? BY : -1;
        const double *ra = si(fa), *rb = fb >= 0 ? si(fb) : nullptr;
        const double ca = sh(ra), cb = rb ? sh(rb) : 0.0;
        T *o2a = nullptr, *o2b = nullptr;
        if (fa == UX && a.d2u) { o2a = f(a.d2udy2, 0); o2b = f(a.d2udy2, 1); }
        if (fa == UZ) {
            o2a = a.d2u ? f(a.d2udy2, 2) : nullptr;
            o2b = a.d2b ? f(a.d2Bdy2, 2) : nullptr;
        }
        if (fa == BX && a.d2b) { o2a = f(a.d2Bdy2, 0); o2b = f(a.d2Bdy2, 1); }
        yr_load<L, T>(A, ra, rb, ca, cb, j, valid);
        if (o2a || o2b) {  // uniform across the block
            // this row's slots of the scratch array: a row of field 2q holds
            // N/2 double2 (FP64: the second half goes to field 2q + 1) or N
            // float2 (FP32)
            C *lo = reinterpret_cast<C *>(a.spec + (size_t)(2 * q) * plane + ro);
            C *hi = sizeof(C) == 16
                        ? reinterpret_cast<C *>(a.spec + (size_t)(2 * q + 1) * plane + ro) - G::N / 2
                        : lo;
            yr_op12<L, T>(tw, A, j, valid, s1, s2, lo, hi, f(a.dudy, fa),
                          fb >= 0 ? f(a.dudy, fb) : nullptr, o2a, o2b);
        } else {
            yr_op<L, T, false>(tw, A, j, valid, s1, f(a.dudy, fa), fb >= 0 ? f(a.dudy, fb) : nullptr);
        }
    }
    if (a.mode != 2) {
        // E = -u x B formed in FP64; d/dy of Ex and Ez.  Ex (out-of-plane
        // family: uz, Bz, Ex, Ey) and Ez (in-plane) never share a transform,
        // so that a field the reference keeps exactly zero (2-D flows) stays
        // exactly zero here too instead of picking up the rounding of its
        // partner: on rows of one CTA each goes through its own real
        // transform (yr_real_pair, the cost of one packed pair); on shorter
        // rows Ex is packed with Ey (whose d/dy is not needed) and Ez alone.
        auto efield = [&](size_t o, double &ex, double &ey, double &ez) {
            const double *u = a.uin + o;
            double ux = u[UX * plane], uy = u[UY * plane], uz = u[UZ * plane];
            double bx = u[BX * plane], by = u[BY * plane], bz = u[BZ * plane];
            ex = uz * by - uy * bz;
            ey = ux * bz - uz * bx;
            ez = uy * bx - ux * by;
        };
        double cx = 0.0, cy = 0.0, cz = 0.0;
        if (MIX && valid) efield(ro, cx, cy, cz);
        if constexpr (G::ROWS == 1 && L >= 5) {
            // Ex and Ez as real rows, side by side (yr_real_pair)
            T *ox = f(a.dEdy, 0), *oz = f(a.dEdy, 2);
            yr_real_pair<L, T>(
                Abase, tw, s1,
                [&](int g, int i) -> T {
                    double ex = 0.0, ey = 0.0, ez = 0.0;
                    if (valid) efield(ro + i, ex, ey, ez);
                    return g == 0 ? (T)(ex - cx) : (T)(ez - cz);
                },
                [&](int g, int i, T v) {
                    if (valid) (g == 0 ? ox : oz)[i] = v;
                });
        } else {
#pragma unroll 4
            for (int m = 0; m < 16; m++) {
                const int i = j + m * G::T_;
                double ex = 0.0, ey = 0.0, ez = 0.0;
                if (valid) efield(ro + i, ex, ey, ez);
                A[fpad(i)] = cmk<C>((T)(ex - cx), (T)(ey - cy));
            }
            yr_op<L, T, false>(tw, A, j, valid, s1, f(a.dEdy, 0), (T *)nullptr);
#pragma unroll 4
            for (int m = 0; m < 16; m++) {
                const int i = j + m * G::T_;
                double ex = 0.0, ey = 0.0, ez = 0.0;
                if (valid) efield(ro + i, ex, ey, ez);
                A[fpad(i)] = cmk<C>((T)(ez - cz), (T)0);
            }
            yr_op<L, T, false>(tw, A, j, valid, s1, f(a.dEdy, 2), (T *)nullptr);
        }
    }

    if (a.mode == 1) return;  // uniform across the grid

    // ---- 2. right-hand side and RK3 update, point by point ------------------
    // (FP64 state and RK3 accumulation in both precisions; the fluxes in T)
    double cc = a.cc, dd = a.dd;
    RhsCoef kc = a.k;
    if (a.dtdev) {
        const double dt = a.dtdev[0];
        cc = a.ccoef * dt;
        dd = a.dcoef * dt;
        if (kc.cleaning == 2) {
            kc.Ch = a.dtdev[1];
            kc.Cp = a.dtdev[2];
        }
    }
    if (valid) {
        const int nv = a.nvar;
        const T *dEdx = reinterpret_cast<const T *>(a.dEdx);
        const T *dEdy = reinterpret_cast<const T *>(a.dEdy);
        const T *dudx = reinterpret_cast<const T *>(a.dudx);
        const T *dudy = reinterpret_cast<const T *>(a.dudy);
        const T *d2udx2 = reinterpret_cast<const T *>(a.d2udx2);
        const T *d2udy2 = reinterpret_cast<const T *>(a.d2udy2);
        const T *d2Bdx2 = reinterpret_cast<const T *>(a.d2Bdx2);
        const T *d2Bdy2 = reinterpret_cast<const T *>(a.d2Bdy2);
#pragma unroll 1
        for (int m = 0; m < 16; m++) {
            const size_t o = ro + j + m * G::T_;
            T u[9], dx[9], dy[9], d2x[6], d2y[6], r[9];
#pragma unroll
            for (int v = 0; v < 9; v++) {
                if (v < nv) {
                    u[v] = (T)a.uin[v * plane + o];
                    dx[v] = dudx[v * plane + o];
                    dy[v] = dudy[v * plane + o];
                } else {
                    u[v] = dx[v] = dy[v] = (T)0;
                }
            }
#pragma unroll
            for (int c = 0; c < 3; c++) {
                d2x[c] = a.k.visc > 0 ? d2udx2[c * plane + o] : (T)0;
                d2y[c] = a.k.visc > 0 ? d2udy2[c * plane + o] : (T)0;
                d2x[3 + c] = a.k.resist > 0 ? d2Bdx2[c * plane + o] : (T)0;
                d2y[3 + c] = a.k.resist > 0 ? d2Bdy2[c * plane + o] : (T)0;
            }
            const T dbx = a.ddivbdx ? (T)a.ddivbdx[o] : (T)0;
            const T dby = a.ddivbdy ? (T)a.ddivbdy[o] : (T)0;
            rhs_point<T>(kc, u, dx, dy, d2x, d2y, dEdx[plane + o], dEdx[2 * plane + o], dEdy[o],
                         dEdy[2 * plane + o], dbx, dby, r);
#pragma unroll
            for (int v = 0; v < 9; v++) {
                if (v < nv) {
                    double rk = a.read_rk ? a.dudtRK[v * plane + o] : 0.0;
                    const double rv = (double)r[v];
                    // the FP64 state: re-read in FP32 mode (an L1 hit), the
                    // value already held in FP64 mode
                    const double ud = MIX ? a.uin[v * plane + o] : (double)u[v];
                    a.uu[v * plane + o] = ud + cc * rv + dd * rk;
                    if (a.write_rk) a.dudtRK[v * plane + o] = rv;
                }
            }
        }
    }
    __syncthreads();  // the updated rows are visible to the whole block

    // ---- 3. spectral y filter of the updated fields, two at a time ----------
    // FP64: the filtered row replaces the row.  FP32: the filter minus the
    // identity is applied to the shifted row and its result added to the
    // FP64 row.
    // the pairs of the derivatives: (ux, uy) (rho, p) (uz, Bz) (Bx, By) [psi]
    const int nfp = a.nvar == 9 ? 5 : 4;
    for (int q = 0; q < nfp; q++) {
        const int v = q == 0 ? UX : q == 1 ? RHO : q == 2 ? UZ : q == 3 ? BX : PSI;
        const int w = q == 0 ? UY : q == 1 ? P : q == 2 ? BZ : q == 3 ? BY : -1;
        double *ra = su(v), *rb = w >= 0 ? su(w) : nullptr;
        const double ca = sh(ra), cb = rb ? sh(rb) : 0.0;
        yr_load<L, T>(A, ra, rb, ca, cb, j, valid);
        if constexpr (MIX)
            yr_op<L, T, true>(tw, A, j, valid, reinterpret_cast<const C *>(a.sfd32), ra, rb);
        else
            yr_op<L, T, false>(tw, A, j, valid, reinterpret_cast<const C *>(a.sf), ra, rb);
    }
}

template <int L, typename T>
static int launch_yrow_l(Ctx *c, const YRArgs &a, double bytes)
{
    using G = YRGeom<L, T>;
    const size_t smem = G::SMEM;
    // the shared-memory attribute, set once per device; contexts on several
    // host threads launch here concurrently
    static std::mutex attr_mu;
    static bool attr_done[64] = {false};
    int dev = 0;
    MHD_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
    {
        std::lock_guard<std::mutex> lock(attr_mu);
        if (!attr_done[dev]) {
            MHD_CUDA_TRY(cudaFuncSetAttribute(yrow_kernel<L, T>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr_done[dev] = true;
        }
    }
    const unsigned grid = (unsigned)((c->nx + G::ROWS - 1) / G::ROWS);
    prof_begin(c, KC_FUSED_Y, bytes);
    yrow_kernel<L, T><<<grid, G::THREADS, smem, c->stream>>>(a);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    return MHDGPU_OK;
}

// Whether the row kernel serves this context (16 <= ny <= 8192).
bool yrow_supported(const Ctx *c) { return c->ny >= 16 && c->ny <= 8192; }

int launch_yrow(Ctx *c, int iRK, int last_stage, int mode)
{
    const mhdgpu_params &p = c->p;
    YRArgs a;
    a.uin = state_ptr(c);
    a.uu = c->arr[MHDGPU_UU];
    a.dudtRK = c->arr[MHDGPU_DUDTRK];
    a.spec = c->arr[MHDGPU_DUDT];  // unused by the fused stage otherwise
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
    a.tw32 = c->ytab32;
    a.s1_32 = c->ytab32 + c->ny;
    a.s2_32 = c->ytab32 + 2 * c->ny;
    a.sfd32 = c->ytab32 + 3 * c->ny;
    a.nx = c->nx;
    a.ny = c->ny;
    a.nvar = c->nvar;
    a.k = RhsCoef{p.adiabaticIdx, p.viscosity, p.resistivity, c->const_diff_divb, c->Ch, c->Cp,
                  p.divBcleaning};
    a.cc = c->cc[iRK];
    a.dd = c->dd[iRK];
    static const double CC[3] = {8.0 / 15.0, 5.0 / 12.0, 0.75};  // rkInit, timeAdvance.c:20-27
    static const double DD[3] = {0.0, -17. / 60., -5. / 12.};
    a.dtdev = c->dev_dt ? c->dscal : nullptr;
    a.ccoef = CC[iRK];
    a.dcoef = DD[iRK];
    a.mode = mode;
    const bool diffuse = p.divBcleaning == 1;
    a.ddivbdx = diffuse ? c->arr[MHDGPU_DDIVBDX] : nullptr;
    a.ddivbdy = diffuse ? c->arr[MHDGPU_DDIVBDY] : nullptr;
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
    if (c->mixed) {
        // the x derivatives are read as floats: half their bytes
        const double b = bytes - (double)c->nx * c->ny * 4.0 * nx_der;
        switch (c->ny) {
        case 16: return launch_yrow_l<4, float>(c, a, b);
        case 32: return launch_yrow_l<5, float>(c, a, b);
        case 64: return launch_yrow_l<6, float>(c, a, b);
        case 128: return launch_yrow_l<7, float>(c, a, b);
        case 256: return launch_yrow_l<8, float>(c, a, b);
        case 512: return launch_yrow_l<9, float>(c, a, b);
        case 1024: return launch_yrow_l<10, float>(c, a, b);
        case 2048: return launch_yrow_l<11, float>(c, a, b);
        case 4096: return launch_yrow_l<12, float>(c, a, b);
        case 8192: return launch_yrow_l<13, float>(c, a, b);
        default: return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
        }
    }
    switch (c->ny) {
    case 16: return launch_yrow_l<4, double>(c, a, bytes);
    case 32: return launch_yrow_l<5, double>(c, a, bytes);
    case 64: return launch_yrow_l<6, double>(c, a, bytes);
    case 128: return launch_yrow_l<7, double>(c, a, bytes);
    case 256: return launch_yrow_l<8, double>(c, a, bytes);
    case 512: return launch_yrow_l<9, double>(c, a, bytes);
    case 1024: return launch_yrow_l<10, double>(c, a, bytes);
    case 2048: return launch_yrow_l<11, double>(c, a, bytes);
    case 4096: return launch_yrow_l<12, double>(c, a, bytes);
    case 8192: return launch_yrow_l<13, double>(c, a, bytes);
    default: return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
    }
}

}  // namespace mhd
