"""GPU: the failure path of the bounded waits, without any GPU fault.

Every TMA wait in the x kernels gives up after a bounded number of SM clocks,
raises the context's status flag and returns.  mhdgpu_selftest_wait runs the
same wait on an mbarrier that nothing completes, with a short limit: the call
must report MHDGPU_ERR_TIMEOUT, and the context must stay usable (the next
steps agree with a fresh context bit for bit).
"""
import time

import numpy as np
import pytest

from mhd2dcfdfftw_open_b200 import ic
from mhd2dcfdfftw_open_b200.solver import Domain, MhdGpuError

pytestmark = pytest.mark.gpu

TIMEOUT = 5  # MHDGPU_ERR_TIMEOUT


def test_wait_runs_out_and_reports_timeout():
    p, uu = ic.orszag_tang(64, 64)
    with Domain(p, uu) as d, Domain(p, uu) as fresh:
        t0 = time.perf_counter()
        rc = d.lib.mhdgpu_selftest_wait(d.h, 50.0)
        elapsed = time.perf_counter() - t0
        assert rc == TIMEOUT
        assert elapsed < 5.0                      # the wait ended by itself
        assert d.lib.mhdgpu_selftest_wait(d.h, 0.0) != 0   # invalid limits are refused
        d.steps(3, 1e-3, fused=True)              # the context still works
        fresh.steps(3, 1e-3, fused=True)
        np.testing.assert_array_equal(d.get("uu"), fresh.get("uu"))
