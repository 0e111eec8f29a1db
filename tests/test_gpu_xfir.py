"""GPU: the chunked x pass of long lines (csrc/xfir.cu) against the
reference and against the cluster x pass it replaces there.

On lines of 1024 rows and more (any length >= 64 with MHDGPU_XN_MIN_NX) the
fused steps take the x filter and the x derivatives from per-chunk Thomas
solves whose inflows are truncated
functionals of the line (weights dropped below 2^-60 of the kept ones).  The
results must meet the same gates as every other path: one RK3 step within
1e-12 per field of the reference built from its own sources, five steps
within 5e-12 of the cluster path (each path is within 1e-12 of the
reference per step) (MHDGPU_NO_XN=1 turns the chunked pass off
for contexts created while it is set), CFL control and hyperbolic cleaning
included, and mixed precision within 1e-5 of FP64.
"""
import os

import numpy as np
import pytest

from conftest import rel_l2, rel_l2_own
from mhd2dcfdfftw_open_b200 import ic
from mhd2dcfdfftw_open_b200.solver import Domain

pytestmark = pytest.mark.gpu


def _run(p, uu, nsteps, dt_fixed, xn=True, mixed=False):
    old = os.environ.pop("MHDGPU_NO_XN", None)
    os.environ["MHDGPU_XN_MIN_NX"] = "64"  # the chunked pass on the short lines too
    if not xn:
        os.environ["MHDGPU_NO_XN"] = "1"
    try:
        with Domain(p, uu) as d:
            if mixed:
                d.set_precision(True)
            dt = d.steps(nsteps, dt_fixed, dt=1e-4, fused=True)
            return d.get("uu"), dt
    finally:
        os.environ.pop("MHDGPU_NO_XN", None)
        os.environ.pop("MHDGPU_XN_MIN_NX", None)
        if old is not None:
            os.environ["MHDGPU_NO_XN"] = old


@pytest.mark.parametrize("nx,ny", [(128, 128), (200, 64), (512, 256), (1024, 64), (1030, 32),
                                   (2048, 16)])
def test_one_step_vs_reference(reference, nx, ny):
    p, uu = ic.alfvenic_turbulence(nx, ny, mmax=min(8, ny // 4))
    reference.setup(p)
    reference.set_state(uu)
    reference.steps(1, 2e-4)
    got, _ = _run(p, uu, 1, 2e-4)
    err = rel_l2_own(got, reference.uu)
    assert err.max() < 1e-12, err


@pytest.mark.parametrize("cfl", [False, True])
def test_steps_match_cluster_path(cfl):
    p, uu = ic.alfvenic_turbulence(2048, 64, mmax=8)
    dtf = 0.0 if cfl else 2e-4
    a, dta = _run(p, uu, 5, dtf, xn=True)
    b, dtb = _run(p, uu, 5, dtf, xn=False)
    # each path is within 1e-12 of the reference per step: 5 steps apart
    assert rel_l2_own(a, b).max() < 5e-12
    assert dta == pytest.approx(dtb, rel=1e-13)


def test_hyperbolic_cleaning_matches_cluster_path():
    p, uu = ic.orszag_tang(1024, 32, di=0.05, divBcleaning=2)
    rng = np.random.default_rng(5)
    uu[8] = 1e-3 * rng.standard_normal(uu.shape[1:])
    a, _ = _run(p, uu, 3, 1e-3, xn=True)
    b, _ = _run(p, uu, 3, 1e-3, xn=False)
    assert rel_l2(a, b).max() < 1e-12


def test_mixed_precision_within_tolerance_of_fp64():
    p, uu = ic.alfvenic_turbulence(1024, 128, mmax=16)
    mix, _ = _run(p, uu, 10, 2e-4, mixed=True)
    f64, _ = _run(p, uu, 10, 2e-4)
    assert rel_l2_own(mix, f64).max() < 1e-5


@pytest.mark.parametrize("cleaning,dt_fixed", [(0, 0.0), (2, 1e-3), (0, 1e-3)])
def test_noise_matches_cluster_path(cleaning, dt_fixed):
    """Seeded noise in a field: the compact filter is far from the identity on
    it, so an x filter applied once too often or too seldom anywhere in the
    step's flow (CFL control and hyperbolic cleaning settle the state before
    calcDt) shows at O(1) instead of hiding below the rounding."""
    p, uu = ic.orszag_tang(1024, 32, di=0.05, divBcleaning=cleaning)
    rng = np.random.default_rng(5)
    uu[0] += 1e-3 * rng.standard_normal(uu.shape[1:])
    if cleaning == 2:
        uu[8] = 1e-3 * rng.standard_normal(uu.shape[1:])
    a, _ = _run(p, uu, 2, dt_fixed, xn=True)
    b, _ = _run(p, uu, 2, dt_fixed, xn=False)
    assert rel_l2_own(a, b).max() < 1e-12
