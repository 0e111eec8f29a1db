// Device helpers shared by the x-direction line kernels (xsolve.cu,
// xline.cu): the compact-scheme right-hand sides of mathlib.c:46-85,
// 176-217 and 309-353, TMA bulk copies with mbarrier completion, and bounded
// waits.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace mhd {

constexpr int XF_EDGE = 160;

// Thomas factor tables of the two distinct matrices (0: derivatives, whose
// first- and second-derivative systems are identical; 1: filter), each
// [3 arrays: m, invB, g][2*EDGE rows: first EDGE, then last EDGE].
struct XFTables {
    const double *edge;   // device, 2 * 3 * 2 * EDGE doubles
    double inner[2][3];
};

struct XFArgs {
    const double *in;     // source array (field 0)
    int in_start;         // first source field
    double *fout;         // filtered-field output (field-indexed), or null: no filter
    double *out1;         // first-derivative output (field-indexed), or null
    double *out2a;        // second-derivative output for fields [d2a_lo, d2a_lo+3)
    double *out2b;        // second-derivative output for fields [d2b_lo, d2b_lo+3)
    int d2a_lo, d2b_lo;
    int single_op;        // -1: the fused program; else one XOp into out1
    int nfields;          // state fields [in_start, in_start + nfields)
    double *outE;         // d/dx of Ey, Ez (2 fields), or null
    XStencil st[3];
    XFTables tb;
    long nx, ny;
    int R, C;
    int hops;             // CTAs whose totals enter a CTA's inflow (C: all)
    double pw[2][2];      // per matrix: (-m)^XL_S, (-g)^XL_S of the interior
    double fa_in, fa_sub; // filter matrix off-diagonals: interior, and rows 0 / n-1
    int *flag;
};


__device__ __forceinline__ double stencil(const XStencil &s, double w0, double w1,
                                          double w2, double w3, double w4, double w5,
                                          double w6, long g, long n)
{
    if (g == 0)
        return s.scale * (s.e0 * w1 + s.e1 * w2 + s.e2 * w3 + s.e3 * w4 + s.e4 * w5);
    if (g == n - 1)
        return s.edge_sign * s.scale *
               (s.e0 * w5 + s.e1 * w4 + s.e2 * w3 + s.e3 * w2 + s.e4 * w1);
    if (s.kind == XOP_D1)
        return s.scale * (s.a * (w4 - w2) + s.b * (w5 - w1) + s.c * (w6 - w0));
    if (s.kind == XOP_D2)
        return s.scale * (s.a * (w4 - 2 * w3 + w2) + s.b * (w5 - 2 * w3 + w1) +
                          s.c * (w6 - 2 * w3 + w0));
    return s.a * w3 + s.b * (w4 + w2) + s.c * (w5 + w1) + s.d * (w6 + w0);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// 2-D tensor-map TMA load of box {x: column, y: row} into shared memory,
// completion counted on an mbarrier (x must be a multiple of 2 for doubles)
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase: `limit` SM clocks at most (about 2 s by
// default), then the error flag is raised and the caller carries on (the data
// are then garbage, which the host reports as MHDGPU_ERR_TIMEOUT).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, int *flag,
                                                  long long limit = 4000000000LL)
{
    long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > limit) {
            if (flag) atomicExch(flag, MHDGPU_ERR_TIMEOUT);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ long wrap(long r, long n)
{
    r %= n;
    return r < 0 ? r + n : r;
}

int launch_xline(Ctx *c, const XFArgs &proto, double bytes);

}  // namespace mhd
