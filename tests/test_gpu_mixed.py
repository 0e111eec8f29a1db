"""GPU: the mixed-precision fused steps (FP32 sweeps, FFT butterflies and
fluxes; FP64 state, RK3 accumulation and compact-scheme right-hand sides)
against the FP64 fused steps, which match the reference to 1e-12.

Tolerance: relative L2 error per field <= 1e-5 after the stated number of
steps (fields with a vanishing norm are scaled by the norm of the state).
"""
import numpy as np
import pytest

from conftest import rel_l2
from mhd2dcfdfftw_open_b200 import ic
from mhd2dcfdfftw_open_b200.solver import Domain, MhdGpuError

pytestmark = pytest.mark.gpu

TOL = 1e-5


def run(p, uu, nsteps, dt, mixed):
    with Domain(p, uu) as d:
        d.set_precision(mixed)
        d.steps(nsteps, dt, fused=True)
        return d.get("uu")


def test_mixed_orszag_tang_1000_steps():
    p, uu = ic.orszag_tang(256, 256, di=0.05)
    ref = run(p, uu, 1000, 1e-3, False)
    mix = run(p, uu, 1000, 1e-3, True)
    err = rel_l2(mix, ref)
    assert err.max() < TOL, err
    assert err.max() > 0.0  # the FP32 path really ran


@pytest.mark.parametrize("nx,ny,nsteps", [(512, 512, 200), (1024, 256, 100), (256, 2048, 50)])
def test_mixed_turbulence(nx, ny, nsteps):
    p, uu = ic.alfvenic_turbulence(nx, ny, mmax=16)
    ref = run(p, uu, nsteps, 2e-4, False)
    mix = run(p, uu, nsteps, 2e-4, True)
    err = rel_l2(mix, ref)
    assert err.max() < TOL, err


def test_mixed_long_lines_clusters():
    # x lines split over a cluster of CTAs (4096 rows: 4 CTAs of 1024)
    p, uu = ic.alfvenic_turbulence(4096, 64, mmax=8)
    ref = run(p, uu, 20, 2e-4, False)
    mix = run(p, uu, 20, 2e-4, True)
    err = rel_l2(mix, ref)
    assert err.max() < TOL, err


def test_mixed_hyperbolic_cleaning():
    p, uu = ic.orszag_tang(128, 128, di=0.05, divBcleaning=2)
    ref = run(p, uu, 100, 1e-3, False)
    mix = run(p, uu, 100, 1e-3, True)
    err = rel_l2(mix, ref)
    assert err.max() < TOL, err


def test_mixed_cfl_dt_matches():
    p, uu = ic.orszag_tang(128, 128, di=0.05)
    with Domain(p, uu) as a, Domain(p, uu) as b:
        b.set_precision(True)
        dta = a.steps(50, 0.0, dt=1e-3, fused=True)
        dtb = b.steps(50, 0.0, dt=1e-3, fused=True)
        assert dtb == pytest.approx(dta, rel=1e-6)
        assert rel_l2(b.get("uu"), a.get("uu")).max() < TOL


def test_mixed_rejections_and_divb_scratch():
    p, uu = ic.orszag_tang(64, 64, divBcleaning=1)
    with Domain(p, uu) as d:
        with pytest.raises(MhdGpuError):
            d.set_precision(True)
    p, uu = ic.orszag_tang(64, 64)
    with Domain(p, uu) as d:
        d.set_precision(True)
        d.steps(2, 1e-3, fused=True)
        with pytest.raises(MhdGpuError):
            d.checkDivB()          # derivative arrays hold FP32 scratch
        d.set_precision(False)
        d.steps(1, 1e-3, fused=True)
        assert np.isfinite(d.checkDivB())
