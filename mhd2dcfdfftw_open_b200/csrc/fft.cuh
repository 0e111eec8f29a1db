// Complex FP64 FFT of one row held in shared memory, for the y-direction
// spectral operators (the reference's FFTW r2c/c2r round trips,
// calcDerivs.c:75-150 and filtering.c:40-94, done here on two real rows at a
// time packed as one complex row).
//
// Stockham auto-sort passes, radix 16 while possible then one radix-8/4/2
// pass, natural order in and out, unnormalised in both directions.  A group
// of T = N/16 threads owns a row; every thread keeps 16 complex values in
// registers per pass.  Element i lives at index i + i/16 of the row buffer:
// with this padding the strided accesses of the passes hit distinct
// shared-memory banks.  Twiddles exp(-2 pi i m / N) come from a table; per
// radix-16 butterfly four are loaded (w, w^2, w^4, w^8) and the others are
// products of at most three of them.
#pragma once

#include <cuda_runtime.h>

namespace mhd {

__device__ __forceinline__ int fpad(int i) { return i + (i >> 4); }

__device__ __forceinline__ double2 cm(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 ca(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cs(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// multiply by -i (forward, SIGN = -1) or +i (inverse, SIGN = +1)
template <int SIGN>
__device__ __forceinline__ double2 cmi(double2 a)
{
    return SIGN < 0 ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x);
}

template <int SIGN>
__device__ __forceinline__ void dft2(double2 &a, double2 &b)
{
    double2 t = a;
    a = ca(t, b);
    b = cs(t, b);
}

// X_k = sum_n v_n exp(SIGN 2 pi i n k / 4)
template <int SIGN>
__device__ __forceinline__ void dft4(double2 &v0, double2 &v1, double2 &v2, double2 &v3)
{
    double2 a0 = ca(v0, v2), a1 = cs(v0, v2), a2 = ca(v1, v3), a3 = cmi<SIGN>(cs(v1, v3));
    v0 = ca(a0, a2);
    v1 = ca(a1, a3);
    v2 = cs(a0, a2);
    v3 = cs(a1, a3);
}

template <int SIGN>
__device__ __forceinline__ void dft8(double2 *v)
{
    // 2 x 4: X[p + 4 s] = sum_q W2^{q s} W8^{q p} (sum_m v[q + 2 m] W4^{m p})
    const double r = 0.70710678118654752440;
    dft4<SIGN>(v[0], v[2], v[4], v[6]);
    dft4<SIGN>(v[1], v[3], v[5], v[7]);
    // twiddles W8^{p} on the odd half: p = 1, 2, 3
    v[3] = cm(v[3], make_double2(r, SIGN * r));
    v[5] = cmi<SIGN>(v[5]);
    v[7] = cm(v[7], make_double2(-r, SIGN * r));
    double2 o[8];
#pragma unroll
    for (int p = 0; p < 4; p++) {
        double2 a = v[2 * p], b = v[2 * p + 1];
        o[p] = ca(a, b);
        o[p + 4] = cs(a, b);
    }
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = o[i];
}

template <int SIGN>
__device__ __forceinline__ void dft16(double2 *v)
{
    // 4 x 4: X[p + 4 s] = sum_q W4^{q s} W16^{q p} (sum_m v[q + 4 m] W4^{m p})
    const double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173;
    const double r = 0.70710678118654752440;
#pragma unroll
    for (int q = 0; q < 4; q++) dft4<SIGN>(v[q], v[q + 4], v[q + 8], v[q + 12]);
    // after the inner DFTs v[q + 4 p] holds term p of column q; twiddle W16^{q p}
    v[5] = cm(v[5], make_double2(c1, SIGN * s1));    // q1 p1
    v[9] = cm(v[9], make_double2(r, SIGN * r));      // q1 p2
    v[13] = cm(v[13], make_double2(s1, SIGN * c1));  // q1 p3
    v[6] = cm(v[6], make_double2(r, SIGN * r));      // q2 p1
    v[10] = cmi<SIGN>(v[10]);                        // q2 p2
    v[14] = cm(v[14], make_double2(-r, SIGN * r));   // q2 p3
    v[7] = cm(v[7], make_double2(s1, SIGN * c1));    // q3 p1
    v[11] = cm(v[11], make_double2(-r, SIGN * r));   // q3 p2
    v[15] = cm(v[15], make_double2(-c1, -SIGN * s1));  // q3 p3: W16^9
    double2 o[16];
#pragma unroll
    for (int p = 0; p < 4; p++) {
        double2 a = v[4 * p], b = v[4 * p + 1], c = v[4 * p + 2], d = v[4 * p + 3];
        dft4<SIGN>(a, b, c, d);
        o[p] = a;
        o[p + 4] = b;
        o[p + 8] = c;
        o[p + 12] = d;
    }
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = o[i];
}

template <int R, int SIGN>
__device__ __forceinline__ void dftr(double2 *v)
{
    if constexpr (R == 16) dft16<SIGN>(v);
    else if constexpr (R == 8) dft8<SIGN>(v);
    else if constexpr (R == 4) dft4<SIGN>(v[0], v[1], v[2], v[3]);
    else dft2<SIGN>(v[0], v[1]);
}

__device__ __forceinline__ double2 twl(const double2 *__restrict__ tw, int m, int sign)
{
    double2 w = __ldg(tw + m);
    if (sign > 0) w.y = -w.y;
    return w;
}

// One Stockham pass of radix R on a row of N points whose sub-transforms have
// length NS: butterfly t < N/R reads elements t + r N/R, multiplies them by
// W_{NS R}^{k r} (k = t mod NS), transforms them and writes element
// (t - k) R + k + r NS.  Thread j of the row's group does butterflies
// j, j + N/16, ...  Two barriers: all reads complete before any write.
template <int N, int R, int NS, int SIGN>
__device__ __forceinline__ void fft_pass(double2 *z, const double2 *__restrict__ tw, int j)
{
    constexpr int T = N / 16;
    constexpr int NB = 16 / R;
    double2 v[NB][R];
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int t = j + b * T;
#pragma unroll
        for (int r = 0; r < R; r++) v[b][r] = z[fpad(t + r * (N / R))];
        if (NS > 1) {
            const int k = t & (NS - 1);
            const int st = k * (N / (NS * R));
            if constexpr (R == 16) {
                double2 w1 = twl(tw, st, SIGN), w2 = twl(tw, 2 * st, SIGN);
                double2 w4 = twl(tw, 4 * st, SIGN), w8 = twl(tw, 8 * st, SIGN);
                double2 w3 = cm(w1, w2), w5 = cm(w1, w4), w6 = cm(w2, w4), w7 = cm(w3, w4);
                v[b][1] = cm(v[b][1], w1);
                v[b][2] = cm(v[b][2], w2);
                v[b][3] = cm(v[b][3], w3);
                v[b][4] = cm(v[b][4], w4);
                v[b][5] = cm(v[b][5], w5);
                v[b][6] = cm(v[b][6], w6);
                v[b][7] = cm(v[b][7], w7);
                v[b][8] = cm(v[b][8], w8);
                v[b][9] = cm(v[b][9], cm(w1, w8));
                v[b][10] = cm(v[b][10], cm(w2, w8));
                v[b][11] = cm(v[b][11], cm(w3, w8));
                v[b][12] = cm(v[b][12], cm(w4, w8));
                v[b][13] = cm(v[b][13], cm(w5, w8));
                v[b][14] = cm(v[b][14], cm(w6, w8));
                v[b][15] = cm(v[b][15], cm(w7, w8));
            } else {
#pragma unroll
                for (int r = 1; r < R; r++) v[b][r] = cm(v[b][r], twl(tw, r * st, SIGN));
            }
        }
        dftr<R, SIGN>(v[b]);
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int t = j + b * T;
        const int k = t & (NS - 1);
        const int base = (t - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) z[fpad(base + r * NS)] = v[b][r];
    }
    __syncthreads();
}

// In-place FFT of the padded row z (N = 2^L >= 16 points) by the N/16 threads
// j = 0..N/16-1 of its group; every thread of the block must call it.
template <int L, int SIGN>
__device__ __forceinline__ void fft_row(double2 *z, const double2 *__restrict__ tw, int j)
{
    constexpr int N = 1 << L;
    static_assert(L >= 4 && L <= 13, "row length 16..8192");
    fft_pass<N, 16, 1, SIGN>(z, tw, j);
    if constexpr (L >= 8) fft_pass<N, 16, 16, SIGN>(z, tw, j);
    if constexpr (L >= 12) fft_pass<N, 16, 256, SIGN>(z, tw, j);
    constexpr int REM = L % 4;
    constexpr int NSR = 1 << (4 * (L / 4));
    if constexpr (REM == 1) fft_pass<N, 2, NSR, SIGN>(z, tw, j);
    if constexpr (REM == 2) fft_pass<N, 4, NSR, SIGN>(z, tw, j);
    if constexpr (REM == 3) fft_pass<N, 8, NSR, SIGN>(z, tw, j);
}

}  // namespace mhd
