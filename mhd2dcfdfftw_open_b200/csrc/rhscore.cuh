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
// d2x/d2y: second derivatives of ux, uy, uz, Bx, By, Bz (unused ones ignored);
// eyx = dEy/dx, ezx = dEz/dx, exy = dEx/dy, ezy = dEz/dy;
// dbx, dby: d(divB)/dx, d(divB)/dy for diffusive cleaning; out: dudt.
__device__ __forceinline__ void rhs_point(const RhsCoef &k, const double *u, const double *dx,
                                          const double *dy, const double *d2x, const double *d2y,
                                          double eyx, double ezx, double exy, double ezy,
                                          double dbx, double dby, double *out)
{
    const double rho = u[RHO], ux = u[UX], uy = u[UY];
    const double bx = u[BX], by = u[BY], bz = u[BZ], pr = u[P];
    double divU = dx[UX] + dy[UY];
    double divB = dx[BX] + dy[BY];
    double jx = dy[BZ];
    double jy = -dx[BZ];
    double jz = dx[BY] - dy[BX];
    double r_rho = -rho * divU - ux * dx[RHO] - uy * dy[RHO];
    double r_ux = -ux * dx[UX] - uy * dy[UX] - dx[P] / rho + jy * bz / rho - jz * by / rho;
    double r_uy = -ux * dx[UY] - uy * dy[UY] - dy[P] / rho + jz * bx / rho - jx * bz / rho;
    double r_uz = -ux * dx[UZ] - uy * dy[UZ] + jx * by / rho - jy * bx / rho;
    double r_bx = -ezy;
    double r_by = ezx;
    double r_bz = exy - eyx;
    double r_p = -ux * dx[P] - uy * dy[P] - k.gamma * pr * divU;
    if (k.cleaning == 2) {
        r_ux = r_ux - divB * bx;
        r_uy = r_uy - divB * by;
        r_uz = r_uz - divB * bz;
        r_bx = r_bx - dx[PSI];
        r_by = r_by - dy[PSI];
        out[PSI] = -k.Ch * k.Ch * (divB + u[PSI] / k.Cp / k.Cp);
    }
    if (k.visc > 0) {
        r_ux = r_ux + k.visc / rho * (d2x[0] + d2y[0]);
        r_uy = r_uy + k.visc / rho * (d2x[1] + d2y[1]);
        r_uz = r_uz + k.visc / rho * (d2x[2] + d2y[2]);
    }
    if (k.resist > 0) {
        r_bx = r_bx + k.resist * (d2x[3] + d2y[3]);
        r_by = r_by + k.resist * (d2x[4] + d2y[4]);
        r_bz = r_bz + k.resist * (d2x[5] + d2y[5]);
    }
    if (k.cleaning == 1) {
        r_bx = r_bx + k.cdiff * dbx;
        r_by = r_by + k.cdiff * dby;
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
