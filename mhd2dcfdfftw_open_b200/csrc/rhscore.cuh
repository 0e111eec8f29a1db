// Right-hand side of the MHD equations at one point: calcRHSInnerPoint
// (calcRHS.c:77-161) followed by addSourceTerm (calcRHS.c:498-544), with the
// reference's order of operations.  Shared by the operator path
// (pointwise.cu) and the fused y pass (yrow.cu).
#pragma once

#include "common.cuh"

namespace mhd {

struct RhsCoef {
    double gamma, visc, resist, cdiff, Ch, Cp;
    int cleaning;
};

// u, dx, dy: NVAR values of the state and its first derivatives;
// T: the arithmetic type (double, or float for the mixed-precision stage);
// d2x/d2y: second derivatives of ux, uy, uz, Bx, By, Bz (unused ones ignored);
// eyx = dEy/dx, ezx = dEz/dx, exy = dEx/dy, ezy = dEz/dy;
// dbx, dby: d(divB)/dx, d(divB)/dy for diffusive cleaning; out: dudt.
template <typename T>
__device__ __forceinline__ void rhs_point(const RhsCoef &k, const T *u, const T *dx, const T *dy,
                                          const T *d2x, const T *d2y, T eyx, T ezx, T exy, T ezy,
                                          T dbx, T dby, T *out)
{
    const T gamma = (T)k.gamma, visc = (T)k.visc, resist = (T)k.resist, cdiff = (T)k.cdiff;
    const T Ch = (T)k.Ch, Cp = (T)k.Cp;
    const T rho = u[RHO], ux = u[UX], uy = u[UY];
    const T bx = u[BX], by = u[BY], bz = u[BZ], pr = u[P];
    T divU = dx[UX] + dy[UY];
    T divB = dx[BX] + dy[BY];
    T jx = dy[BZ];
    T jy = -dx[BZ];
    T jz = dx[BY] - dy[BX];
    T r_rho = -rho * divU - ux * dx[RHO] - uy * dy[RHO];
    T r_ux = -ux * dx[UX] - uy * dy[UX] - dx[P] / rho + jy * bz / rho - jz * by / rho;
    T r_uy = -ux * dx[UY] - uy * dy[UY] - dy[P] / rho + jz * bx / rho - jx * bz / rho;
    T r_uz = -ux * dx[UZ] - uy * dy[UZ] + jx * by / rho - jy * bx / rho;
    T r_bx = -ezy;
    T r_by = ezx;
    T r_bz = exy - eyx;
    T r_p = -ux * dx[P] - uy * dy[P] - gamma * pr * divU;
    if (k.cleaning == 2) {
        r_ux = r_ux - divB * bx;
        r_uy = r_uy - divB * by;
        r_uz = r_uz - divB * bz;
        r_bx = r_bx - dx[PSI];
        r_by = r_by - dy[PSI];
        out[PSI] = -Ch * Ch * (divB + u[PSI] / Cp / Cp);
    }
    if (k.visc > 0) {
        r_ux = r_ux + visc / rho * (d2x[0] + d2y[0]);
        r_uy = r_uy + visc / rho * (d2x[1] + d2y[1]);
        r_uz = r_uz + visc / rho * (d2x[2] + d2y[2]);
    }
    if (k.resist > 0) {
        r_bx = r_bx + resist * (d2x[3] + d2y[3]);
        r_by = r_by + resist * (d2x[4] + d2y[4]);
        r_bz = r_bz + resist * (d2x[5] + d2y[5]);
    }
    if (k.cleaning == 1) {
        r_bx = r_bx + cdiff * dbx;
        r_by = r_by + cdiff * dby;
    }
    out[RHO] = r_rho;
    out[UX] = r_ux;
    out[UY] = r_uy;
    out[UZ] = r_uz;
    out[BX] = r_bx;
    out[BY] = r_by;
    out[BZ] = r_bz;
    out[P] = r_p;
}

}  // namespace mhd
