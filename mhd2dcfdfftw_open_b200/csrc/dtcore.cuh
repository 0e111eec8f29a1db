// Per-cell CFL speeds of calcDt (timeAdvance.c:55-105), shared by the
// context path (pointwise.cu) and the allocation-free entry (noalloc.cu).
#pragma once

#include "common.cuh"

namespace mhd {

struct DtArgs {
    const double *uu;
    long plane, ny;
    double gamma, dx, dy, di, resist, visc;
    int hall;
    double *part;
};

// The reference's MAX and MIN (macros.h:26-27): a comparison and a choice,
// so that a NaN operand comes out exactly as it does there (MAX(a, b) is b
// whenever either is NaN; fmax/fmin would instead drop the NaN).
__device__ __forceinline__ double ref_max(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double ref_min(double a, double b) { return a < b ? a : b; }

// cmaxx, cmaxy of one cell (timeAdvance.c:55-105)
__device__ __forceinline__ void cell_speeds(const DtArgs &a, long o, double &cmaxx, double &cmaxy)
{
    const long plane = a.plane;
    const double *u = a.uu;
    double rho = u[RHO * plane + o];
    double csound2 = a.gamma * u[P * plane + o] / rho;
    double sr = sqrt(rho);
    double cax = u[BX * plane + o] / sr, cay = u[BY * plane + o] / sr, caz = u[BZ * plane + o] / sr;
    double ca2 = cax * cax + cay * cay + caz * caz;
    double cms2 = csound2 + ca2;
    double cnsx2 = sqrt(ref_max(cms2 * cms2 - 4 * csound2 * cax * cax, 0.));
    double cnsy2 = sqrt(ref_max(cms2 * cms2 - 4 * csound2 * cay * cay, 0.));
    const double s2 = sqrt(2.);
    double cfx = sqrt(cms2 + cnsx2) / s2, cfy = sqrt(cms2 + cnsy2) / s2;
    double csx = sqrt(ref_max(cms2 - cnsx2, 0.)) / s2, csy = sqrt(ref_max(cms2 - cnsy2, 0.)) / s2;
    double ux = u[UX * plane + o], uy = u[UY * plane + o];
    double t = ref_max(fabs(ux), fabs(ux - cax));
    t = ref_max(fabs(ux - csx), t);
    t = ref_max(fabs(ux - cfx), t);
    t = ref_max(fabs(ux + cax), t);
    t = ref_max(fabs(ux + csx), t);
    cmaxx = ref_max(fabs(ux + cfx), t);
    t = ref_max(fabs(uy), fabs(uy - cay));
    t = ref_max(fabs(uy - csy), t);
    t = ref_max(fabs(uy - cfy), t);
    t = ref_max(fabs(uy + cay), t);
    t = ref_max(fabs(uy + csy), t);
    cmaxy = ref_max(fabs(uy + cfy), t);
    if (a.hall == 1) {
        double ch = a.di / ref_min(a.dx, a.dy) / rho *
                    ref_max(fabs(u[BX * plane + o]), ref_max(fabs(u[BY * plane + o]), fabs(u[BZ * plane + o])));
        cmaxx = ref_max(cmaxx, ch);
        cmaxy = ref_max(cmaxy, ch);
    }
}

// MIN(dtx, dty) of one cell with the diffusive limits (timeAdvance.c:114-129)
__device__ __forceinline__ double cell_dt(const DtArgs &a, long o)
{
    double cx, cy;
    cell_speeds(a, o, cx, cy);
    double dtx = a.dx / cx, dty = a.dy / cy;
    if (a.resist > 0) {
        dtx = ref_min(dtx, a.dx * a.dx / a.resist);
        dty = ref_min(dty, a.dy * a.dy / a.resist);
    }
    if (a.visc > 0) {
        dtx = ref_min(dtx, a.dx * a.dx / a.visc);
        dty = ref_min(dty, a.dy * a.dy / a.visc);
    }
    return ref_min(dtx, dty);
}

// The reference's minimum over the cells is a running minimum in loop order
// (timeAdvance.c:47, 131-134): dtmin = -1, then per cell
// `if (dtmin < 0 || v < dtmin) dtmin = v`.  A negative dtmin (a cell with
// rho < 0 under the Hall speed) is replaced by the next cell whatever it is;
// a NaN that lands there (or in the first cell) stays for good.  So the
// result is NaN if a NaN cell comes first or right after a negative cell;
// otherwise, after the last negative cell L, it is v(L) when L is the last
// cell and the minimum of the cells after L (NaN cells skipped) otherwise;
// with no negative cell, the minimum of all cells.
//
// In parallel: per cell, the NaN-skipping minimum, the largest index of a
// negative cell and a flag for a NaN cell whose predecessor is negative (or
// which is the first cell) are reduced in any order (dt_cell_fold); the final
// block resolves the rare states with a negative cell by a second pass over
// the cells after L (dt_resolve).
struct DtFold {
    double mn, lastneg, nanflag;
};

__device__ __forceinline__ void dt_cell_fold(const DtArgs &a, long o, DtFold &f)
{
    const double v = cell_dt(a, o);
    if (v != v) {
        const double prev = o == 0 ? -1.0 : cell_dt(a, o - 1);
        if (prev < 0) f.nanflag = 1.0;
        return;
    }
    f.mn = fmin(f.mn, v);
    if (v < 0) f.lastneg = fmax(f.lastneg, (double)o);
}

// The running minimum from the folded (mn, lastneg, nanflag); every thread of
// the block calls it (a second pass over the cells after the last negative
// one runs on the whole block); `red` is shared scratch of 32 doubles.
__device__ __forceinline__ double dt_resolve(const DtArgs &a, double mn, double lastneg, double nanflag, double *red)
{
    if (nanflag > 0) return __longlong_as_double(0x7ff8000000000000LL);  // NaN
    if (lastneg < 0) return mn;
    const long L = (long)lastneg;
    if (L == a.plane - 1) return cell_dt(a, L);
    double m = INFINITY;
    for (long o = L + 1 + threadIdx.x; o < a.plane; o += blockDim.x) m = fmin(m, cell_dt(a, o));
    for (int s = 16; s > 0; s >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, s));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    double r = INFINITY;
    for (int w = 0; w < (int)(blockDim.x / 32); w++) r = fmin(r, red[w]);
    return r;
}

}  // namespace mhd
