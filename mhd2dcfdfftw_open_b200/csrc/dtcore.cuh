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
    double cnsx2 = sqrt(fmax(cms2 * cms2 - 4 * csound2 * cax * cax, 0.));
    double cnsy2 = sqrt(fmax(cms2 * cms2 - 4 * csound2 * cay * cay, 0.));
    const double s2 = sqrt(2.);
    double cfx = sqrt(cms2 + cnsx2) / s2, cfy = sqrt(cms2 + cnsy2) / s2;
    double csx = sqrt(fmax(cms2 - cnsx2, 0.)) / s2, csy = sqrt(fmax(cms2 - cnsy2, 0.)) / s2;
    double ux = u[UX * plane + o], uy = u[UY * plane + o];
    double t = fmax(fabs(ux), fabs(ux - cax));
    t = fmax(fabs(ux - csx), t);
    t = fmax(fabs(ux - cfx), t);
    t = fmax(fabs(ux + cax), t);
    t = fmax(fabs(ux + csx), t);
    cmaxx = fmax(fabs(ux + cfx), t);
    t = fmax(fabs(uy), fabs(uy - cay));
    t = fmax(fabs(uy - csy), t);
    t = fmax(fabs(uy - cfy), t);
    t = fmax(fabs(uy + cay), t);
    t = fmax(fabs(uy + csy), t);
    cmaxy = fmax(fabs(uy + cfy), t);
    if (a.hall == 1) {
        double ch = a.di / fmin(a.dx, a.dy) / rho *
                    fmax(fabs(u[BX * plane + o]), fmax(fabs(u[BY * plane + o]), fabs(u[BZ * plane + o])));
        cmaxx = fmax(cmaxx, ch);
        cmaxy = fmax(cmaxy, ch);
    }
}

// min(dtx, dty) of one cell with the diffusive limits (timeAdvance.c:114-129)
__device__ __forceinline__ double cell_dt(const DtArgs &a, long o)
{
    double cx, cy;
    cell_speeds(a, o, cx, cy);
    double dtx = a.dx / cx, dty = a.dy / cy;
    if (a.resist > 0) {
        dtx = fmin(dtx, a.dx * a.dx / a.resist);
        dty = fmin(dty, a.dy * a.dy / a.resist);
    }
    if (a.visc > 0) {
        dtx = fmin(dtx, a.dx * a.dx / a.visc);
        dty = fmin(dty, a.dy * a.dy / a.visc);
    }
    return fmin(dtx, dty);
}

}  // namespace mhd
