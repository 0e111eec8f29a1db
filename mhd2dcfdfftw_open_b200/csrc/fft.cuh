// Complex FFT of one row held in shared memory, for the y-direction spectral
// operators (the reference's FFTW r2c/c2r round trips, calcDerivs.c:75-150
// and filtering.c:40-94, done here on two real rows at a time packed as one
// complex row).  Generic in the complex type: double2 (FP64) or float2.
//
// Stockham auto-sort passes, natural order in and out, unnormalised in both
// directions: one radix-2/4/8 pass first when log2 N is not a multiple of 4
// (sub-transform length 1, so it needs no twiddles), then radix-16 passes.
// A group of T = N/16 threads owns a row; every thread keeps 16 complex
// values in registers per pass.  Element i lives at index i + i/16 of the
// row buffer: with this padding the strided accesses of the passes hit
// distinct shared-memory banks.  Twiddles exp(-2 pi i m / N) come from a
// table; per radix-16 butterfly four are loaded (w, w^2, w^4, w^8) and the
// others are products of at most three of them.
#pragma once

#include <cuda_runtime.h>

namespace mhd {

__device__ __forceinline__ int fpad(int i) { return i + (i >> 4); }

template <typename C>
using creal_t = decltype(C{}.x);

template <typename C>
__device__ __forceinline__ C cmk(creal_t<C> x, creal_t<C> y)
{
    C r;
    r.x = x;
    r.y = y;
    return r;
}
template <typename C>
__device__ __forceinline__ C cm(C a, C b)
{
    return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C>
__device__ __forceinline__ C ca(C a, C b) { return cmk<C>(a.x + b.x, a.y + b.y); }
template <typename C>
__device__ __forceinline__ C cs(C a, C b) { return cmk<C>(a.x - b.x, a.y - b.y); }
// multiply by -i (forward, SIGN = -1) or +i (inverse, SIGN = +1)
template <int SIGN, typename C>
__device__ __forceinline__ C cmi(C a)
{
    return SIGN < 0 ? cmk<C>(a.y, -a.x) : cmk<C>(-a.y, a.x);
}

template <int SIGN, typename C>
__device__ __forceinline__ void dft2(C &a, C &b)
{
    C t = a;
    a = ca(t, b);
    b = cs(t, b);
}

// X_k = sum_n v_n exp(SIGN 2 pi i n k / 4)
template <int SIGN, typename C>
__device__ __forceinline__ void dft4(C &v0, C &v1, C &v2, C &v3)
{
    C a0 = ca(v0, v2), a1 = cs(v0, v2), a2 = ca(v1, v3), a3 = cmi<SIGN>(cs(v1, v3));
    v0 = ca(a0, a2);
    v1 = ca(a1, a3);
    v2 = cs(a0, a2);
    v3 = cs(a1, a3);
}

template <int SIGN, typename C>
__device__ __forceinline__ void dft8(C *v)
{
    // 2 x 4: X[p + 4 s] = sum_q W2^{q s} W8^{q p} (sum_m v[q + 2 m] W4^{m p})
    using R = creal_t<C>;
    const R r = (R)0.70710678118654752440;
    dft4<SIGN>(v[0], v[2], v[4], v[6]);
    dft4<SIGN>(v[1], v[3], v[5], v[7]);
    // twiddles W8^{p} on the odd half: p = 1, 2, 3
    v[3] = cm(v[3], cmk<C>(r, SIGN * r));
    v[5] = cmi<SIGN>(v[5]);
    v[7] = cm(v[7], cmk<C>(-r, SIGN * r));
    C o[8];
#pragma unroll
    for (int p = 0; p < 4; p++) {
        C a = v[2 * p], b = v[2 * p + 1];
        o[p] = ca(a, b);
        o[p + 4] = cs(a, b);
    }
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = o[i];
}

template <int SIGN, typename C>
__device__ __forceinline__ void dft16(C *v)
{
    // 4 x 4: X[p + 4 s] = sum_q W4^{q s} W16^{q p} (sum_m v[q + 4 m] W4^{m p})
    using R = creal_t<C>;
    const R c1 = (R)0.92387953251128675613, s1 = (R)0.38268343236508977173;
    const R r = (R)0.70710678118654752440;
#pragma unroll
    for (int q = 0; q < 4; q++) dft4<SIGN>(v[q], v[q + 4], v[q + 8], v[q + 12]);
    // after the inner DFTs v[q + 4 p] holds term p of column q; twiddle W16^{q p}
    v[5] = cm(v[5], cmk<C>(c1, SIGN * s1));    // q1 p1
    v[9] = cm(v[9], cmk<C>(r, SIGN * r));      // q1 p2
    v[13] = cm(v[13], cmk<C>(s1, SIGN * c1));  // q1 p3
    v[6] = cm(v[6], cmk<C>(r, SIGN * r));      // q2 p1
    v[10] = cmi<SIGN>(v[10]);                  // q2 p2
    v[14] = cm(v[14], cmk<C>(-r, SIGN * r));   // q2 p3
    v[7] = cm(v[7], cmk<C>(s1, SIGN * c1));    // q3 p1
    v[11] = cm(v[11], cmk<C>(-r, SIGN * r));   // q3 p2
    v[15] = cm(v[15], cmk<C>(-c1, -SIGN * s1));  // q3 p3: W16^9
    // outer DFTs over q for each p; results in place, then transposed
#pragma unroll
    for (int p = 0; p < 4; p++) dft4<SIGN>(v[4 * p], v[4 * p + 1], v[4 * p + 2], v[4 * p + 3]);
    // X[p + 4 s] = v[4 p + s]: transpose the 4 x 4 block
#pragma unroll
    for (int p = 0; p < 4; p++)
#pragma unroll
        for (int s = p + 1; s < 4; s++) {
            C t = v[4 * p + s];
            v[4 * p + s] = v[4 * s + p];
            v[4 * s + p] = t;
        }
}

template <int R, int SIGN, typename C>
__device__ __forceinline__ void dftr(C *v)
{
    if constexpr (R == 16) dft16<SIGN>(v);
    else if constexpr (R == 8) dft8<SIGN>(v);
    else if constexpr (R == 4) dft4<SIGN>(v[0], v[1], v[2], v[3]);
    else dft2<SIGN>(v[0], v[1]);
}

template <int SIGN, typename C>
__device__ __forceinline__ C twl(const C *__restrict__ tw, int m)
{
    C w = __ldg(tw + m);
    if (SIGN > 0) w.y = -w.y;
    return w;
}

// One Stockham pass of radix R on a row of N points whose sub-transforms have
// length NS: butterfly t < N/R reads elements t + r N/R, multiplies them by
// W_{NS R}^{k r} (k = t mod NS), transforms them and writes element
// (t - k) R + k + r NS.  Thread j of the row's group does butterflies
// j, j + N/16, ...  Two barriers: all reads complete before any write.
// Twiddled passes (NS > 1) are radix 16 only.
template <int N, int R, int NS, int SIGN, typename C, int TWS = 1>
__device__ __forceinline__ void fft_pass(C *z, const C *__restrict__ tw, int j)
{
    constexpr int T = N / 16;
    constexpr int NB = 16 / R;
    static_assert(NS == 1 || R == 16, "twiddled passes are radix 16");
    C v[NB][R];
    // element j + T m (m = b + r 16/R) sits at fpad(j) + m (T + T/16) when T
    // is a multiple of 16: one base address for all loads
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int t = j + b * T;
#pragma unroll
        for (int r = 0; r < R; r++) {
            if constexpr (T % 16 == 0)
                v[b][r] = z[fpad(j) + (b + r * (16 / R)) * (T + T / 16)];
            else
                v[b][r] = z[fpad(t + r * (N / R))];
        }
    }
    if constexpr (NS > 1) {
        const int k = j & (NS - 1);
        const int st = k * (N / (NS * 16)) * TWS;
        // v[r + 8] takes W^{r+8} = W^r W^8: first the W^8 factor, then W^r
        // for both halves, so that few twiddles are live at a time
        const C w8 = twl<SIGN>(tw, 8 * st);
#pragma unroll
        for (int r = 8; r < 16; r++) v[0][r] = cm(v[0][r], w8);
        const C w1 = twl<SIGN>(tw, st), w2 = twl<SIGN>(tw, 2 * st), w4 = twl<SIGN>(tw, 4 * st);
        const C w3 = cm(w1, w2);
        v[0][1] = cm(v[0][1], w1);
        v[0][9] = cm(v[0][9], w1);
        v[0][2] = cm(v[0][2], w2);
        v[0][10] = cm(v[0][10], w2);
        v[0][3] = cm(v[0][3], w3);
        v[0][11] = cm(v[0][11], w3);
        v[0][4] = cm(v[0][4], w4);
        v[0][12] = cm(v[0][12], w4);
        const C w5 = cm(w1, w4);
        v[0][5] = cm(v[0][5], w5);
        v[0][13] = cm(v[0][13], w5);
        const C w6 = cm(w2, w4);
        v[0][6] = cm(v[0][6], w6);
        v[0][14] = cm(v[0][14], w6);
        const C w7 = cm(w3, w4);
        v[0][7] = cm(v[0][7], w7);
        v[0][15] = cm(v[0][15], w7);
    }
#pragma unroll
    for (int b = 0; b < NB; b++) dftr<R, SIGN>(v[b]);
    __syncthreads();
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int t = j + b * T;
        const int k = t & (NS - 1);
        const int base = (t - k) * R + k;
#pragma unroll
        // with NS and R powers of two, k < NS and k + r NS never carrying
        // into bit 4 beyond r NS: fpad(base + r NS) = fpad(base) + r NS + (r NS >> 4)
        for (int r = 0; r < R; r++) z[fpad(base) + r * NS + ((r * NS) >> 4)] = v[b][r];
    }
    __syncthreads();
}

// In-place FFT of the padded row z (N = 2^L >= 16 points) by the N/16 threads
// j = 0..N/16-1 of its group; every thread of the block must call it.  The
// twiddle table holds exp(-2 pi i m / (TWS N)) (TWS > 1: a table made for a
// longer row).
template <int L, int SIGN, typename C, int TWS = 1>
__device__ __forceinline__ void fft_row(C *z, const C *__restrict__ tw, int j)
{
    constexpr int N = 1 << L;
    static_assert(L >= 4 && L <= 13, "row length 16..8192");
    constexpr int REM = L % 4;
    constexpr int R0 = 1 << REM;  // the twiddle-free first pass (1: none)
    if constexpr (REM == 1) fft_pass<N, 2, 1, SIGN, C, TWS>(z, tw, j);
    if constexpr (REM == 2) fft_pass<N, 4, 1, SIGN, C, TWS>(z, tw, j);
    if constexpr (REM == 3) fft_pass<N, 8, 1, SIGN, C, TWS>(z, tw, j);
    fft_pass<N, 16, R0, SIGN, C, TWS>(z, tw, j);
    if constexpr (L >= 8) fft_pass<N, 16, R0 * 16, SIGN, C, TWS>(z, tw, j);
    if constexpr (L >= 12) fft_pass<N, 16, R0 * 256, SIGN, C, TWS>(z, tw, j);
}

}  // namespace mhd
