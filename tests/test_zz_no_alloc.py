"""GPU: the allocation-free time-step entry point, mhdgpu_calc_dt_noalloc.

It serves callers that cannot allocate device memory when they need a step
size: a framework whose pool allocator owns the device's memory, or a service
that fixes its memory footprint at start-up.  Its scratch is a fixed device
array inside the library.  This test calls it through the C ABI twice in a
row, on two different states, and checks each result against the context
entry point mhdgpu_calc_dt (which allocates its scratch with the context),
within the tolerance the other calcDt tests use.  It sits in its own file,
collected last, and runs the same alone or after the other tests.
"""
import ctypes

import mhd_oracle as O
import numpy as np
import pytest

from mhd2dcfdfftw_open_b200 import ic
from mhd2dcfdfftw_open_b200.config import CParams
from mhd2dcfdfftw_open_b200.solver import Domain, load_library

pytestmark = pytest.mark.gpu


def _entry():
    lib = load_library()
    f = lib.mhdgpu_calc_dt_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.POINTER(CParams), ctypes.c_double, ctypes.c_void_p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


@pytest.mark.parametrize("cleaning", [0, 2])
def test_noalloc_dt_matches_context_entry_on_two_calls(cleaning):
    import torch

    f = _entry()
    p, uu0 = ic.orszag_tang(96, 64, di=0.05, divBcleaning=cleaning)
    rng = np.random.default_rng(3)
    states = [uu0, uu0 + 0.05 * rng.standard_normal(uu0.shape) * (np.arange(uu0.shape[0]) != 0)[:, None, None]]
    cp = CParams.from_params(p)
    with Domain(p) as d:
        out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda:0")
        for k, state in enumerate(states):  # two calls in a row
            d.set("uu", state)
            dt0 = 0.0 if k == 0 else 1e-3
            want_dt = d.calcDt(dt0)
            want_ch, want_cp = d.cleaning_speeds()
            rc = f(d.device_ptr("uu"), ctypes.byref(cp), dt0, out.data_ptr(), d.stream_handle())
            assert rc == 0
            d.synchronize()
            got = out.cpu().numpy()
            assert got[0] == pytest.approx(want_dt, rel=1e-14)
            # and directly against the oracle's calcDt (timeAdvance.c:38-153)
            odt, och, ocp = O.calcDt(p, state, dt0)
            assert got[0] == pytest.approx(odt, rel=1e-14)
            if cleaning == 2:
                assert got[1] == pytest.approx(och, rel=1e-14)
                assert got[2] == pytest.approx(ocp, rel=1e-14)
            if cleaning == 2:
                assert got[1] == pytest.approx(want_ch, rel=1e-14)
                assert got[2] == pytest.approx(want_cp, rel=1e-14)
            else:
                assert got[1] == 0.0 and got[2] == 0.0


def test_noalloc_rejects_grids_beyond_its_scratch():
    f = _entry()
    p, _ = ic.orszag_tang(16, 16)
    p.nx, p.ny = 16384, 4096  # 67M cells > 33,554,432
    cp = CParams.from_params(p)
    # rejected on the host before any launch; the pointers are never touched
    assert f(ctypes.c_void_p(16), ctypes.byref(cp), 0.0, ctypes.c_void_p(16), None) == 1


@pytest.mark.parametrize("bad", [[(1, 17, 23, np.nan)], [(1, 0, 0, np.nan)],
                                 [(0, 5, 5, -1.0), (7, 9, 9, -2.0)],
                                 [(0, 5, 5, -1.0), (1, 5, 6, np.nan)],
                                 [(0, 63, 63, -1.0)]])
def test_noalloc_dt_on_broken_states_matches_context_entry(bad):
    """NaN or negative density in the state: both entries follow the
    reference's calcDt (its MAX/MIN per cell and its running minimum, which a
    negative cell resets), so they agree with each other and with the
    oracle's restatement (pinned to the reference in test_oracle.py)."""
    import torch

    f = _entry()
    p, uu = ic.orszag_tang(64, 64, di=0.05)
    uu = uu.copy()
    for v, i, j, x in bad:
        uu[v, i, j] = x
    cp = CParams.from_params(p)
    want_o = O.calcDt(p, uu, 1e-3)[0]
    with Domain(p) as d:
        d.set("uu", uu)
        want = d.calcDt(1e-3)
        out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda:0")
        assert f(d.device_ptr("uu"), ctypes.byref(cp), 1e-3, out.data_ptr(), d.stream_handle()) == 0
        d.synchronize()
        got = float(out[0].item())
    if np.isnan(want_o):
        assert np.isnan(got) and np.isnan(want)
    else:
        assert got == pytest.approx(want, rel=1e-14)
        assert got == pytest.approx(want_o, rel=1e-14)
