"""CPU oracle: a numpy restatement of the reference solver's per-step hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module; only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may use it, and only as the checker.

Parity is pinned: ``tests/test_oracle.py`` compares this restatement with the
reference itself (its own C sources compiled unmodified into
``oracle/_ref/libmhdref.so`` against single-rank MPI/FFTW-API shims, see
``oracle/Makefile``) and with the golden fixtures in ``tests/golden/`` that the
reference produced (``tests/golden/make_golden.py``).

Layout: a state ``uu`` is ``[NVAR][nx][ny]`` (``macros.h:4-24``); x-lines have
stride ny, y is contiguous.  Every function restates one reference routine for
the periodic x boundary at one MPI rank (the only configuration the workloads
use), with the 2-point halos of ``parallel.c:13-24`` written as periodic
wrap-around.  The stencils keep the reference's expression order, so the
finite-difference parts agree with the reference to the last bit; the spectral
parts use numpy's FFT instead of FFTW and agree to rounding.
"""
from __future__ import annotations

import math

import numpy as np

PI = math.acos(-1.0)  # parameter.h:14

# ---------------------------------------------------------------------------
# Scheme constants: parameter.h:23-56 and initializeCFDSchemes
# (initialize.c:572-631).  alphaSub2 is initialised from ALPHASUB1
# (initialize.c:33); both are 0.
# ---------------------------------------------------------------------------
alphaInner1 = 0.375
alphaSub1 = 0.0
alphaInner2 = 0.375
alphaSub2 = 0.0
alphaInnerF = 0.49
alphaSubF = 0.95

aInner1 = (alphaInner1 + 9.) / 6.
bInner1 = (32 * alphaInner1 - 9.) / 15.
cInner1 = (-3. * alphaInner1 + 1) / 10.
aInner2 = (6. - 9. * alphaInner2) / 4.
bInner2 = (-3. + 24. * alphaInner2) / 5.
cInner2 = (2. - 11. * alphaInner2) / 20.
aSub1 = (1. - alphaSub1) / 12.
bSub1 = (3. * alphaSub1 - 4.) / 6.
cSub1 = -3. / 2. * alphaSub1
dSub1 = (4. + 5. * alphaSub1) / 6.
eSub1 = (3. * alphaSub1 - 1.) / 12.
aSub2 = -(1. + alphaSub2) / 12.
bSub2 = (alphaSub2 + 4.) / 3.
cSub2 = (alphaSub2 - 5.) / 2.
dSub2 = (4. - 5. * alphaSub2) / 3.
eSub2 = (11. * alphaSub2 - 1.) / 12.
aInnerF = (11. + 10. * alphaInnerF) / 16.
bInnerF = (15. + 34. * alphaInnerF) / 32.
cInnerF = (-3. + 6. * alphaInnerF) / 16.
dInnerF = (1. - 2. * alphaInnerF) / 32.
aSubF = (alphaSubF - 1.) / 16.
bSubF = (1 - alphaSubF) / 4.
cSubF = (3. * alphaSubF + 5.) / 8.
dSubF = (3. * alphaSubF + 1.) / 4.
eSubF = (alphaSubF - 1.) / 16.

# RK3 coefficients (timeAdvance.c:11-16, 20-27)
CC = (8.0 / 15.0, 5.0 / 12.0, 0.75)
DD = (0.0, -17. / 60., -5. / 12.)
CR_DIVB_CLEANING = 0.18  # divBcleaning.c:4

RHO, UX, UY, UZ, BX, BY, BZ, P, PSI = range(9)


def tri_matrix(n: int, alpha_inner: float, alpha_sub: float):
    """Diagonals of the x-direction system for a periodic x boundary
    (initTriMatrixCFD1st/2nd/Filter, initialize.c:636-654, 713-731, 790-808):
    unit diagonal, alpha_inner off the diagonal, alpha_sub on the two edge
    rows.  The system is NOT cyclic."""
    low = np.full(n - 1, alpha_inner)
    low[n - 2] = alpha_sub
    cent = np.ones(n)
    up = np.full(n - 1, alpha_inner)
    up[0] = alpha_sub
    return low, cent, up


def thomas(A, B, C, R):
    """tridiagonalSolver (mathlib.c:8-30), vectorised over trailing axes of R:
    forward elimination m = A[i-1]/B[i-1] then back substitution."""
    n = R.shape[0]
    B = B.astype(np.float64).copy()
    R = R.copy()
    for i in range(1, n):
        m = A[i - 1] / B[i - 1]
        B[i] = B[i] - m * C[i - 1]
        R[i] = R[i] - m * R[i - 1]
    X = np.empty_like(R)
    X[n - 1] = R[n - 1] / B[n - 1]
    for i in range(n - 2, -1, -1):
        X[i] = (R[i] - C[i] * X[i + 1]) / B[i]
    return X


def _ext(a):
    """a[N, ...] extended by the periodic 2-point halos on both sides:
    index k of the result is row k-2 (parallel.c:13-24 at one rank)."""
    return np.concatenate([a[-2:], a, a[:2]], axis=0)


def deriv_cfd1(a, DX):
    """derivCFD1st periodic branch (mathlib.c:46-85) along axis 0."""
    N = a.shape[0]
    e = _ext(a)
    A = lambda i: e[i + 2]  # noqa: E731  (row i, halos at -2..-1 and N..N+1)
    B = np.empty_like(a)
    B[0] = 1 / DX * (aSub1 * A(-2) + bSub1 * A(-1) + cSub1 * A(0) + dSub1 * A(1) + eSub1 * A(2))
    i = np.arange(1, N - 1)
    B[1:N - 1] = 1 / DX * (aInner1 / 2 * (e[i + 3] - e[i + 1]) + bInner1 / 4 * (e[i + 4] - e[i])
                           + cInner1 / 6 * (e[i + 5] - e[i - 1]))
    B[N - 1] = -1 / DX * (aSub1 * A(N + 1) + bSub1 * A(N) + cSub1 * A(N - 1)
                          + dSub1 * A(N - 2) + eSub1 * A(N - 3))
    return thomas(*tri_matrix(N, alphaInner1, alphaSub1), B)


def deriv_cfd2(a, DX):
    """derivCFD2nd periodic branch (mathlib.c:176-217) along axis 0."""
    N = a.shape[0]
    DX2 = DX * DX
    e = _ext(a)
    A = lambda i: e[i + 2]  # noqa: E731
    B = np.empty_like(a)
    B[0] = 1 / DX2 * (aSub2 * A(-2) + bSub2 * A(-1) + cSub2 * A(0) + dSub2 * A(1) + eSub2 * A(2))
    i = np.arange(1, N - 1)
    c = e[i + 2]
    B[1:N - 1] = 1 / DX2 * (aInner2 * (e[i + 3] - 2 * c + e[i + 1])
                            + bInner2 / 4 * (e[i + 4] - 2 * c + e[i])
                            + cInner2 / 9 * (e[i + 5] - 2 * c + e[i - 1]))
    B[N - 1] = 1 / DX2 * (aSub2 * A(N + 1) + bSub2 * A(N) + cSub2 * A(N - 1)
                          + dSub2 * A(N - 2) + eSub2 * A(N - 3))
    return thomas(*tri_matrix(N, alphaInner2, alphaSub2), B)


def filter_cfd(a):
    """filterCFD periodic branch (mathlib.c:309-353) along axis 0."""
    N = a.shape[0]
    e = _ext(a)
    A = lambda i: e[i + 2]  # noqa: E731
    B = np.empty_like(a)
    B[0] = aSubF * A(-2) + bSubF * A(-1) + cSubF * A(0) + dSubF * A(1) + eSubF * A(2)
    i = np.arange(1, N - 1)
    B[1:N - 1] = (aInnerF * e[i + 2] + bInnerF / 2 * (e[i + 3] + e[i + 1])
                  + cInnerF / 2 * (e[i + 4] + e[i]) + dInnerF / 2 * (e[i + 5] + e[i - 1]))
    B[N - 1] = aSubF * A(N + 1) + bSubF * A(N) + cSubF * A(N - 1) + dSubF * A(N - 2) + eSubF * A(N - 3)
    return thomas(*tri_matrix(N, alphaInnerF, alphaSubF), B)


# ---------------------------------------------------------------------------
# Whole-array operators (calcDerivs.c, filtering.c) on [nv][nx][ny] arrays.
# ---------------------------------------------------------------------------
def derivX(arr, dx):
    """derivX (calcDerivs.c:9-39): compact first derivative of every x-line."""
    return np.moveaxis(deriv_cfd1(np.moveaxis(arr, -2, 0), dx), 0, -2)


def derivXX(arr, dx):
    """derivXX (calcDerivs.c:41-72)."""
    return np.moveaxis(deriv_cfd2(np.moveaxis(arr, -2, 0), dx), 0, -2)


def filteringX(arr):
    """filteringX (filtering.c:9-37): compact filter of every x-line."""
    return np.moveaxis(filter_cfd(np.moveaxis(arr, -2, 0)), 0, -2)


def _rfft(a):
    return np.fft.rfft(a, axis=-1)


def _irfft(F, n):
    # unnormalised inverse, like FFTW's c2r; the imaginary parts of the DC and
    # Nyquist bins are ignored, as FFTW's c2r does
    F = F.copy()
    F[..., 0] = F[..., 0].real
    if n % 2 == 0:
        F[..., -1] = F[..., -1].real
    return np.fft.irfft(F, n=n, axis=-1, norm="forward")


def derivY(arr, Ly):
    """derivY (calcDerivs.c:75-109): r2c, (re, im) <- (-im, re)*2pi/Ly*k/ny,
    c2r.  c2r drops the imaginary part of the Nyquist bin, so the Nyquist
    component of the first derivative vanishes."""
    ny = arr.shape[-1]
    F = _rfft(arr)
    ik = np.arange(F.shape[-1], dtype=np.float64)
    re, im = F.real, F.imag
    nre = -im * 2 * PI / Ly * ik / ny
    nim = re * 2 * PI / Ly * ik / ny
    return _irfft(nre + 1j * nim, ny)


def derivYY(arr, Ly):
    """derivYY (calcDerivs.c:114-150): multiply by -(2pi/Ly*k)^2/ny; the
    Nyquist bin is kept."""
    ny = arr.shape[-1]
    F = _rfft(arr)
    ik = np.arange(F.shape[-1], dtype=np.float64)
    f = (2 * PI / Ly * ik) ** 2
    return _irfft(-F.real * f / ny + 1j * (-F.imag * f / ny), ny)


def filt_y(ny, afy=0.45):
    """Spectral filter transfer filtY[k] (initialize.c:161-177)."""
    nky = ny // 2 + 1
    aj = (5.0 + 6.0 * afy) / 8.0
    bj = (1.0 + 2.0 * afy) / 2.0
    cj = -(1.0 - 2 * afy) / 8.0
    k = np.arange(nky, dtype=np.float64)
    w = 2. * PI * k / ny
    return (aj + bj * np.cos(w) + cj * np.cos(2 * w)) / (1 + 2 * afy * np.cos(w))


def filteringY(arr, option=1):
    """filteringY (filtering.c:40-94); option 1 (the default,
    initialize.c:43) multiplies by filtY[k]/ny, option 0 cuts k > ny/3."""
    ny = arr.shape[-1]
    F = _rfft(arr)
    if option == 1:
        f = filt_y(ny)
        F = F / ny * f
    else:
        k = np.arange(F.shape[-1])
        F = np.where(k <= math.floor(ny / 3), F / ny, 0)
    return _irfft(F, ny)


def filtering(uu):
    """filtering (filtering.c:98-102): x filter, then y filter."""
    return filteringY(filteringX(uu))


# ---------------------------------------------------------------------------
# Pointwise operators (calcRHS.c) and time integration (timeAdvance.c).
# ---------------------------------------------------------------------------
def calcEfield(uu):
    """E = -u x B (calcRHS.c:24-43)."""
    E = np.empty((3,) + uu.shape[1:])
    E[0] = uu[UZ] * uu[BY] - uu[UY] * uu[BZ]
    E[1] = uu[UX] * uu[BZ] - uu[UZ] * uu[BX]
    E[2] = uu[UY] * uu[BX] - uu[UX] * uu[BY]
    return E


def calcDivB(dudx, dudy):
    """calcDivB (calcRHS.c:13-22)."""
    return dudx[BX] + dudy[BY]


def calcRHS(p, uu, dudx, dudy, dEdx, dEdy, d2udx2=None, d2udy2=None,
            d2Bdx2=None, d2Bdy2=None, ddivBdx=None, ddivBdy=None,
            Ch=0.0, Cp=0.0):
    """calcRHSInnerPoint (calcRHS.c:77-161) on the whole periodic domain
    (calcRHS.c:52-55), then addSourceTerm (calcRHS.c:498-544)."""
    dudt = np.zeros_like(uu)
    divU = dudx[UX] + dudy[UY]
    divB_point = dudx[BX] + dudy[BY]
    currentX = dudy[BZ]
    currentY = -dudx[BZ]
    currentZ = dudx[BY] - dudy[BX]
    rho = uu[RHO]
    dudt[RHO] = -uu[RHO] * divU - uu[UX] * dudx[RHO] - uu[UY] * dudy[RHO]
    dudt[UX] = (-uu[UX] * dudx[UX] - uu[UY] * dudy[UX] - dudx[P] / rho
                + currentY * uu[BZ] / rho - currentZ * uu[BY] / rho)
    dudt[UY] = (-uu[UX] * dudx[UY] - uu[UY] * dudy[UY] - dudy[P] / rho
                + currentZ * uu[BX] / rho - currentX * uu[BZ] / rho)
    dudt[UZ] = (-uu[UX] * dudx[UZ] - uu[UY] * dudy[UZ]
                + currentX * uu[BY] / rho - currentY * uu[BX] / rho)
    dudt[BX] = -dEdy[2]
    dudt[BY] = dEdx[2]
    dudt[BZ] = dEdy[0] - dEdx[1]
    dudt[P] = -uu[UX] * dudx[P] - uu[UY] * dudy[P] - p.adiabaticIdx * uu[P] * divU
    if p.divBcleaning == 2:
        dudt[UX] = dudt[UX] - divB_point * uu[BX]
        dudt[UY] = dudt[UY] - divB_point * uu[BY]
        dudt[UZ] = dudt[UZ] - divB_point * uu[BZ]
        dudt[BX] = dudt[BX] - dudx[PSI]
        dudt[BY] = dudt[BY] - dudy[PSI]
        dudt[PSI] = -Ch * Ch * (divB_point + uu[PSI] / Cp / Cp)
    if p.viscosity > 0:
        for c in range(3):
            dudt[UX + c] = dudt[UX + c] + p.viscosity / uu[RHO] * (d2udx2[c] + d2udy2[c])
    if p.resistivity > 0:
        for c in range(3):
            dudt[BX + c] = dudt[BX + c] + p.resistivity * (d2Bdx2[c] + d2Bdy2[c])
    if p.divBcleaning == 1:
        cd = p.const_diff_divb
        dudt[BX] = dudt[BX] + cd * ddivBdx
        dudt[BY] = dudt[BY] + cd * ddivBdy
    return dudt


def rkExecute(uu, dudt, dudtRK, iRK, dt):
    """rkExecute (timeAdvance.c:29-36) with rkInit's coefficients
    (timeAdvance.c:20-27); returns (uu_new, dudtRK_new)."""
    c = CC[iRK] * dt
    d = DD[iRK] * dt
    return uu + c * dudt + d * dudtRK, dudt.copy()


def MAX(a, b):
    """The reference's MAX (macros.h:26): b whenever a > b is false, which
    includes a NaN on either side."""
    return np.where(a > b, a, b)


def MIN(a, b):
    """The reference's MIN (macros.h:27)."""
    return np.where(a < b, a, b)


def cell_speeds(p, uu):
    """Per-cell cmaxx, cmaxy of calcDt (timeAdvance.c:50-105), with the
    reference's MAX/MIN so that NaN cells come out as they do there."""
    g = p.adiabaticIdx
    with np.errstate(invalid="ignore", divide="ignore"):
        rho = uu[RHO]
        csound2 = g * uu[P] / rho
        sr = np.sqrt(rho)
        cax = uu[BX] / sr
        cay = uu[BY] / sr
        caz = uu[BZ] / sr
        ca2 = cax * cax + cay * cay + caz * caz
        cms2 = csound2 + ca2
        cnsx2 = np.sqrt(MAX(cms2 * cms2 - 4 * csound2 * cax * cax, 0.))
        cnsy2 = np.sqrt(MAX(cms2 * cms2 - 4 * csound2 * cay * cay, 0.))
        cfx = np.sqrt(cms2 + cnsx2) / np.sqrt(2.)
        cfy = np.sqrt(cms2 + cnsy2) / np.sqrt(2.)
        csx = np.sqrt(MAX(cms2 - cnsx2, 0.)) / np.sqrt(2.)
        csy = np.sqrt(MAX(cms2 - cnsy2, 0.)) / np.sqrt(2.)
        ux, uy = uu[UX], uu[UY]
        cmaxx = MAX(np.abs(ux), np.abs(ux - cax))
        for t in (np.abs(ux - csx), np.abs(ux - cfx), np.abs(ux + cax), np.abs(ux + csx),
                  np.abs(ux + cfx)):
            cmaxx = MAX(t, cmaxx)
        cmaxy = MAX(np.abs(uy), np.abs(uy - cay))
        for t in (np.abs(uy - csy), np.abs(uy - cfy), np.abs(uy + cay), np.abs(uy + csy),
                  np.abs(uy + cfy)):
            cmaxy = MAX(t, cmaxy)
        if p.Hall == 1:
            ch = p.di / min(p.dx, p.dy) / rho * MAX(np.abs(uu[BX]),
                                                    MAX(np.abs(uu[BY]), np.abs(uu[BZ])))
            cmaxx = MAX(cmaxx, ch)
            cmaxy = MAX(cmaxy, ch)
    return cmaxx, cmaxy


def cell_dt(p, uu):
    """MIN(dtx, dty) per cell with the diffusive limits (timeAdvance.c:114-129)."""
    cmaxx, cmaxy = cell_speeds(p, uu)
    with np.errstate(invalid="ignore", divide="ignore"):
        dtx = p.dx / cmaxx
        dty = p.dy / cmaxy
        if p.resistivity > 0:
            dtx = MIN(dtx, p.dx * p.dx / p.resistivity)
            dty = MIN(dty, p.dy * p.dy / p.resistivity)
        if p.viscosity > 0:
            dtx = MIN(dtx, p.dx * p.dx / p.viscosity)
            dty = MIN(dty, p.dy * p.dy / p.viscosity)
        return MIN(dtx, dty), cmaxx, cmaxy


def running_min(v):
    """The reference's minimum over the cells in loop order
    (timeAdvance.c:47, 131-134): dtmin = -1, then per cell
    `if (dtmin < 0 || v < dtmin) dtmin = v`.  A negative dtmin is replaced by
    the next cell whatever it is, NaN included (and a NaN dtmin never
    changes again).  Hence: NaN if a NaN cell comes first or right after a
    negative cell; else, after the last negative cell, that cell itself if it
    is the last, or the minimum of the cells after it (NaN cells skipped)."""
    v = np.asarray(v, dtype=np.float64)
    nan = np.isnan(v)
    neg = v < 0
    after_neg = np.concatenate(([True], neg[:-1]))
    if np.any(nan & after_neg):
        return float("nan")
    if not neg.any():
        return float(np.nanmin(v)) if not nan.all() else float("nan")
    last = int(np.flatnonzero(neg)[-1])
    if last == len(v) - 1:
        return float(v[last])
    return float(np.nanmin(v[last + 1:]))


def calcDt(p, uu, dt0):
    """calcDt (timeAdvance.c:38-153).  Returns (dt, Ch, Cp); with hyperbolic
    cleaning Ch is max(cmaxx, cmaxy) of the LAST cell of the loop
    (timeAdvance.c:107-112) and Cp = sqrt(Cr*Ch) (divBcleaning.c:7-10).
    The minimum over the cells is the reference's running minimum
    (running_min)."""
    cdt, cmaxx, cmaxy = cell_dt(p, uu)
    dtmin = running_min(cdt.ravel()) * p.cfl
    dt = dtmin if (dt0 < 0.98 * dtmin or dt0 > 1.02 * dtmin) else dt0
    Ch = Cp = 0.0
    if p.divBcleaning == 2:
        Ch = float(MAX(cmaxx[-1, -1], cmaxy[-1, -1]))
        Cp = math.sqrt(CR_DIVB_CLEANING * Ch)
    return dt, Ch, Cp


class State:
    """The oracle's copy of the reference globals that persist across calls."""

    def __init__(self, p, uu):
        self.p = p
        self.uu = np.array(uu, dtype=np.float64, copy=True)
        self.dudtRK = np.zeros_like(self.uu)
        self.Ch = 0.0
        self.Cp = 0.0
        self.dudx = self.dudy = None


def stage(s: State, iRK: int, dt: float):
    """One RK3 stage in the call order of mhd.c:154-199."""
    p, uu = s.p, s.uu
    dx, Ly = p.dx, p.Ly
    dudx = derivX(uu, dx)
    dudy = derivY(uu, Ly)
    d2udx2 = d2udy2 = d2Bdx2 = d2Bdy2 = ddivBdx = ddivBdy = None
    if p.viscosity > 0:
        d2udx2 = derivXX(uu[1:4], dx)
        d2udy2 = derivYY(uu[1:4], Ly)
    if p.Hall == 1 or p.resistivity > 0:
        d2Bdx2 = derivXX(uu[4:7], dx)
        d2Bdy2 = derivYY(uu[4:7], Ly)
    if p.divBcleaning == 1:
        divB = calcDivB(dudx, dudy)
        ddivBdx = derivX(divB[None], dx)[0]
        ddivBdy = derivY(divB[None], Ly)[0]
    E = calcEfield(uu)
    dEdx = derivX(E, dx)
    dEdy = derivY(E, Ly)
    dudt = calcRHS(p, uu, dudx, dudy, dEdx, dEdy, d2udx2, d2udy2, d2Bdx2,
                   d2Bdy2, ddivBdx, ddivBdy, s.Ch, s.Cp)
    s.uu, s.dudtRK = rkExecute(uu, dudt, s.dudtRK, iRK, dt)
    s.uu = filtering(s.uu)
    s.dudx, s.dudy = dudx, dudy


def steps(s: State, nsteps: int, dt_fixed: float, dt: float = 0.0):
    """nsteps RK3 steps as the harness ref_steps (oracle/ref_harness.c)."""
    p = s.p
    if dt_fixed > 0:
        if p.divBcleaning == 2:
            _, s.Ch, s.Cp = calcDt(p, s.uu, dt_fixed)
        dt = dt_fixed
    else:
        dt, s.Ch, s.Cp = calcDt(p, s.uu, dt)
    s.dudtRK[:] = 0
    for _ in range(nsteps):
        for iRK in range(3):
            stage(s, iRK, dt)
        if dt_fixed > 0:
            if p.divBcleaning == 2:
                _, s.Ch, s.Cp = calcDt(p, s.uu, dt_fixed)
            dt = dt_fixed
        else:
            dt, s.Ch, s.Cp = calcDt(p, s.uu, dt)
        s.dudtRK[:] = 0
    return dt


def check_divb(s: State) -> float:
    """max|dudx[BX] + dudy[BY]| from the last stage's derivatives
    (checkDivB, mhd.c:342-367)."""
    return float(np.max(np.abs(s.dudx[BX] + s.dudy[BY])))


def energy(p, uu) -> float:
    """Total energy sum(rho|u|^2/2 + p/(gamma-1) + |B|^2/2) dx dy."""
    kin = 0.5 * uu[RHO] * (uu[UX] ** 2 + uu[UY] ** 2 + uu[UZ] ** 2)
    mag = 0.5 * (uu[BX] ** 2 + uu[BY] ** 2 + uu[BZ] ** 2)
    th = uu[P] / (p.adiabaticIdx - 1.0)
    return float(np.sum(kin + mag + th) * p.dx * p.dy)


def cross_helicity(p, uu) -> float:
    """sum(u . B) dx dy."""
    return float(np.sum(uu[UX] * uu[BX] + uu[UY] * uu[BY] + uu[UZ] * uu[BZ]) * p.dx * p.dy)
