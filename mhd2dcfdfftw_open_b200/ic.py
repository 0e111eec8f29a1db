"""Seeded initial conditions and job parameters for the solver's workloads.

The reference hard-codes its initial conditions in ``usrInitialize.c:13-400``
(test case 5 is active); none of them is one of the workloads below, so these
generators are this project's own.  Every generator returns
``(InputParams, uu)`` with ``uu`` shaped ``[NVAR][nx][ny]`` in the
reference's variable order (rho, ux, uy, uz, Bx, By, Bz, p; ``macros.h:4-12``)
on the grid ``x_i = i*dx``, ``y_j = j*dy`` (``initialize.c:145-152``).

Workloads
---------
* ``orszag_tang``: periodic [0, 2pi)^2, gamma = 5/3, rho = gamma^2, p = gamma,
  u = (-sin y, sin x, 0), B = (-sin y, sin 2x, 0).
* ``alfvenic_turbulence``: box 20pi x 20pi, rho = 1, B0 = 1 along x,
  beta = 0.5 (p = 0.25), seeded random-phase Alfvenic fluctuations
  dv = dB on integer mode pairs 1 <= |m| <= 32.  "Perpendicular to B0" is
  read as *transverse to k and incompressible*: each mode carries
  ``A_k [ (z x k_hat) cos(k.x + phi1) + z_hat cos(k.x + phi2) ]``, which is
  divergence free and has all three components.  Shell amplitude
  ``A_k ~ |m|^(-5/3) / sqrt(modes in the shell)``, rescaled so that the rms of
  |dB| is 0.5 (relative to B0 = 1).
* ``parametric_decay``: box 16pi x 4pi, B0 = 1 along x, rho = 1 + U(-1e-3, 1e-3),
  beta = 0.3 (p = 0.15), circularly polarised pump of mode 8 along x with
  amplitude 0.2: dBy = 0.2 cos kx, dBz = 0.2 sin kx, du = -dB.
* ``ensemble_jobs`` / ``serving_requests``: seeded job lists for the batched
  and serving forms.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .config import InputParams

RHO, UX, UY, UZ, BX, BY, BZ, P, PSI = range(9)


def _grid(p: InputParams):
    x = np.arange(p.nx, dtype=np.float64) * p.dx
    y = np.arange(p.ny, dtype=np.float64) * p.dy
    return np.meshgrid(x, y, indexing="ij")


def orszag_tang(nx=256, ny=256, di=0.0, eta=1e-4, nu=1e-4, Hall=1,
                divBcleaning=0, cfl=0.3):
    g = 5.0 / 3.0
    p = InputParams(boundaryTypeX=0, cfl=cfl, Tmax=1.0, dtOut=0.1, nx=nx, ny=ny,
                    Lx=2 * math.pi, Ly=2 * math.pi, adiabaticIdx=g, Hall=Hall,
                    di=di, resistivity=eta, viscosity=nu,
                    divBcleaning=divBcleaning, outDivB=0).normalized()
    X, Y = _grid(p)
    uu = np.zeros(p.state_shape())
    g = p.adiabaticIdx
    uu[RHO] = g * g
    uu[UX] = -np.sin(Y)
    uu[UY] = np.sin(X)
    uu[BX] = -np.sin(Y)
    uu[BY] = np.sin(2 * X)
    uu[P] = g
    return p, uu


def _synth(p: InputParams, modes, coef, phase):
    """sum_m coef_m cos(k_m . x + phase_m) on the grid, by one inverse FFT."""
    F = np.zeros((p.nx, p.ny), dtype=np.complex128)
    mx = modes[:, 0] % p.nx
    my = modes[:, 1] % p.ny
    c = 0.5 * coef * np.exp(1j * phase)
    np.add.at(F, (mx, my), c)
    np.add.at(F, ((-modes[:, 0]) % p.nx, (-modes[:, 1]) % p.ny), np.conj(c))
    return np.real(np.fft.ifft2(F)) * (p.nx * p.ny)


def alfvenic_turbulence(nx=4096, ny=4096, seed=1, di=0.1, eta=2e-4, nu=2e-4,
                        mmax=32, rms=0.5, Hall=1, cfl=0.3, Lx=20 * math.pi,
                        Ly=20 * math.pi):
    p = InputParams(boundaryTypeX=0, cfl=cfl, Tmax=1.0, dtOut=0.1, nx=nx, ny=ny,
                    Lx=Lx, Ly=Ly, adiabaticIdx=5.0 / 3.0, Hall=Hall, di=di,
                    resistivity=eta, viscosity=nu, divBcleaning=0,
                    outDivB=0).normalized()
    rng = np.random.default_rng(seed)
    # half plane of integer mode pairs: my > 0, or my == 0 and mx > 0
    ms = []
    for my in range(0, mmax + 1):
        for mx in range(-mmax, mmax + 1):
            if my == 0 and mx <= 0:
                continue
            r = math.hypot(mx, my)
            if 1 <= r <= mmax:
                ms.append((mx, my))
    modes = np.array(ms, dtype=np.int64)
    mag = np.hypot(modes[:, 0], modes[:, 1])
    shell = np.rint(mag).astype(np.int64)
    count = np.bincount(shell)
    amp = mag ** (-5.0 / 3.0) / np.sqrt(count[shell])
    phi1 = rng.uniform(0, 2 * np.pi, len(modes))
    phi2 = rng.uniform(0, 2 * np.pi, len(modes))
    kx = 2 * np.pi * modes[:, 0] / p.Lx
    ky = 2 * np.pi * modes[:, 1] / p.Ly
    kn = np.hypot(kx, ky)
    ex, ey = -ky / kn, kx / kn  # z x k_hat
    dbx = _synth(p, modes, amp * ex, phi1)
    dby = _synth(p, modes, amp * ey, phi1)
    dbz = _synth(p, modes, amp, phi2)
    scale = rms / math.sqrt(float(np.mean(dbx ** 2 + dby ** 2 + dbz ** 2)))
    dbx *= scale
    dby *= scale
    dbz *= scale
    uu = np.zeros(p.state_shape())
    uu[RHO] = 1.0
    uu[UX], uu[UY], uu[UZ] = dbx, dby, dbz
    uu[BX] = 1.0 + dbx
    uu[BY] = dby
    uu[BZ] = dbz
    uu[P] = 0.25
    return p, uu


def parametric_decay(nx=8192, ny=2048, seed=3, di=0.05, eta=1e-4, nu=1e-4,
                     amp=0.2, mode=8, Hall=1, cfl=0.3):
    p = InputParams(boundaryTypeX=0, cfl=cfl, Tmax=1.0, dtOut=0.1, nx=nx, ny=ny,
                    Lx=16 * math.pi, Ly=4 * math.pi, adiabaticIdx=5.0 / 3.0,
                    Hall=Hall, di=di, resistivity=eta, viscosity=nu,
                    divBcleaning=0, outDivB=0).normalized()
    rng = np.random.default_rng(seed)
    X, _ = _grid(p)
    k = 2 * np.pi * mode / p.Lx
    uu = np.zeros(p.state_shape())
    uu[RHO] = 1.0 + rng.uniform(-1e-3, 1e-3, (p.nx, p.ny))
    uu[BX] = 1.0
    uu[BY] = amp * np.cos(k * X)
    uu[BZ] = amp * np.sin(k * X)
    uu[UY] = -uu[BY]
    uu[UZ] = -uu[BZ]
    uu[P] = 0.15
    return p, uu


ENSEMBLE_SIZES = ((128, 128), (256, 128), (256, 256), (512, 256), (512, 512),
                  (1024, 512), (1024, 1024))
SERVING_SIZES = ((128, 128), (256, 256), (512, 512), (1024, 1024), (2048, 2048))


@dataclasses.dataclass
class Job:
    """One simulation job: grid, physics and step count."""

    job_id: int
    nx: int
    ny: int
    generator: str  # "orszag_tang" | "alfvenic_turbulence"
    di: float
    eta: float
    steps: int
    seed: int
    arrival: float = 0.0
    cfl: float = 0.3

    def build(self):
        if self.generator == "orszag_tang":
            return orszag_tang(self.nx, self.ny, di=self.di, eta=self.eta,
                               nu=self.eta, Hall=1, cfl=self.cfl)
        return alfvenic_turbulence(self.nx, self.ny, seed=self.seed, di=self.di,
                                   eta=self.eta, nu=self.eta, Hall=1,
                                   cfl=self.cfl, mmax=min(32, self.nx // 4, self.ny // 4))


def ensemble_jobs(n=64, seed=4, steps=500):
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n):
        nx, ny = ENSEMBLE_SIZES[int(rng.integers(len(ENSEMBLE_SIZES)))]
        s = int(rng.integers(1 << 30))
        gen = "orszag_tang" if s % 2 == 0 else "alfvenic_turbulence"
        di = float(rng.uniform(0.0, 0.1))
        eta = float(10 ** rng.uniform(-4, -3))
        jobs.append(Job(i, nx, ny, gen, di, eta, steps, s))
    return jobs


def serving_requests(n=2000, seed=5, rate=20.0, steps_lo=100, steps_hi=2000):
    rng = np.random.default_rng(seed)
    w = np.array([1.0 / (a * b) for a, b in SERVING_SIZES])
    w /= w.sum()
    t = 0.0
    jobs = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate))
        nx, ny = SERVING_SIZES[int(rng.choice(len(SERVING_SIZES), p=w))]
        s = int(rng.integers(1 << 30))
        gen = "orszag_tang" if s % 2 == 0 else "alfvenic_turbulence"
        di = float(rng.uniform(0.0, 0.1))
        eta = float(10 ** rng.uniform(-4, -3))
        steps = int(rng.integers(steps_lo, steps_hi + 1))
        jobs.append(Job(i, nx, ny, gen, di, eta, steps, s, arrival=t))
    return jobs
