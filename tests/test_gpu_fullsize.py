"""GPU at the bench's full sizes: the Alfvenic-turbulence workload at
4096 x 4096 and the parametric-decay workload at 8192 x 2048.

* One RK3 step of the fused FP64 path against the reference's own C code
  (built at one rank) on the 4096^2 workload: <= 1e-12 relative L2 per field,
  the plain form's one-step gate, plus energy and cross helicity at 1e-12.
* Size-independent properties on both: the fused path equals the operator
  path (both on the GPU) to 1e-12 after three steps, and the mixed-precision
  path stays within 1e-5 of FP64.
"""
import numpy as np
import pytest

import mhd_oracle as O
from conftest import rel_l2
from mhd2dcfdfftw_open_b200 import ic
from mhd2dcfdfftw_open_b200.solver import Domain

pytestmark = pytest.mark.gpu


def test_turbulence_4096_one_step_vs_reference(reference):
    p, uu = ic.alfvenic_turbulence(4096, 4096)
    reference.setup(p)
    reference.set_state(uu)
    reference.steps(1, 2e-4)
    ru = reference.uu.copy()
    with Domain(p, uu) as d:
        d.steps(1, 2e-4, fused=True)
        gu = d.get("uu")
    err = rel_l2(gu, ru)
    assert err.max() < 1e-12, err
    assert O.energy(p, gu) == pytest.approx(O.energy(p, ru), rel=1e-12)
    assert O.cross_helicity(p, gu) == pytest.approx(O.cross_helicity(p, ru), rel=1e-12)


@pytest.mark.parametrize("workload", ["turbulence", "parametric"])
def test_full_size_fused_equals_operators_and_mixed_stays_close(workload):
    if workload == "turbulence":
        p, uu = ic.alfvenic_turbulence(4096, 4096)
        dt = 2e-4
    else:
        p, uu = ic.parametric_decay(8192, 2048)
        dt = 5e-4
    with Domain(p, uu) as d:
        d.steps(3, dt)                      # operator path
        ops = d.get("uu")
        d.set("uu", uu)
        d.steps(3, dt, fused=True)          # fused FP64
        fused = d.get("uu")
        d.set("uu", uu)
        d.set_precision(True)
        d.steps(3, dt, fused=True)          # fused mixed precision
        mixed = d.get("uu")
    assert rel_l2(fused, ops).max() < 1e-12
    err = rel_l2(mixed, fused)
    assert err.max() < 1e-5, err
    assert np.all(np.isfinite(mixed))
