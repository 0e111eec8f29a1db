"""GPU: the fused y pass on rows of 8192 points (one CTA of 512 threads per
row, 136 KB of shared memory in FP64) against the reference.

Rows of that length used to fall back to the operator y sequence (eight
launches per stage) and to refuse mixed precision.  Gates as for every other
row length: one RK3 step within 1e-12 per field of the reference built from
its own sources, through the cluster x pass and through the chunked x pass;
mixed precision within 1e-5 of FP64; the out-of-plane fields of a 2-D flow
exactly zero; max |div B| as the reference reports it.
"""
import os

import numpy as np
import pytest

from conftest import rel_l2, rel_l2_own
from mhd2dcfdfftw_open_b200 import ic
from mhd2dcfdfftw_open_b200.solver import Domain

pytestmark = pytest.mark.gpu


def _run(p, uu, nsteps, dt_fixed, mixed=False, chunked=False):
    saved = os.environ.get("MHDGPU_XN_MIN_NX")
    if chunked:
        os.environ["MHDGPU_XN_MIN_NX"] = "64"
    try:
        with Domain(p, uu) as d:
            if mixed:
                d.set_precision(True)
            dt = d.steps(nsteps, dt_fixed, dt=1e-4, fused=True)
            return d.get("uu"), dt, (None if mixed else d.checkDivB())
    finally:
        if saved is None:
            os.environ.pop("MHDGPU_XN_MIN_NX", None)
        else:
            os.environ["MHDGPU_XN_MIN_NX"] = saved


@pytest.mark.parametrize("chunked", [False, True])
def test_one_step_vs_reference(reference, chunked):
    p, uu = ic.alfvenic_turbulence(64, 8192, mmax=8)
    reference.setup(p)
    reference.set_state(uu)
    reference.steps(1, 2e-4)
    rdiv = reference.check_divb()
    got, _, div = _run(p, uu, 1, 2e-4, chunked=chunked)
    assert rel_l2_own(got, reference.uu).max() < 1e-12
    assert div == pytest.approx(rdiv, rel=1e-9, abs=1e-12)


def test_cfl_steps_vs_reference(reference):
    p, uu = ic.orszag_tang(32, 8192, di=0.05)
    reference.setup(p)
    reference.set_state(uu)
    _, rdt = reference.steps(3, 0.0, dt=1e-4)
    got, dt, _ = _run(p, uu, 3, 0.0)
    assert rel_l2(got, reference.uu).max() < 1e-11
    assert dt == pytest.approx(rdt, rel=1e-12)


def test_mixed_precision_within_tolerance_of_fp64():
    p, uu = ic.alfvenic_turbulence(64, 8192, mmax=8)
    mix, _, _ = _run(p, uu, 10, 2e-4, mixed=True)
    f64, _, _ = _run(p, uu, 10, 2e-4)
    assert rel_l2_own(mix, f64).max() < 1e-5


@pytest.mark.parametrize("mixed", [False, True])
def test_out_of_plane_fields_stay_exactly_zero(mixed):
    p, uu = ic.orszag_tang(32, 8192, di=0.05)
    out, _, _ = _run(p, uu, 5, 1e-3, mixed=mixed)
    assert np.all(out[3] == 0.0) and np.all(out[6] == 0.0)
    assert np.isfinite(out).all()
