"""GPU: the fused two-pass stage (mhdgpu_steps_fused) against the reference
and against the operator path, at the same gates as the operator path:
1e-12 per field after one RK3 step, 1e-9 after 100 steps.
"""
import numpy as np
import pytest

import mhd_oracle as O
from conftest import rel_l2
from mhd2dcfdfftw_open_b200 import ic
from mhd2dcfdfftw_open_b200.solver import Domain

pytestmark = pytest.mark.gpu


def run_ref(reference, p, uu, nsteps, dt_fixed):
    reference.setup(p)
    reference.set_state(uu)
    _, dt = reference.steps(nsteps, dt_fixed)
    return reference.uu.copy(), dt


@pytest.mark.parametrize("nx,ny", [(64, 64), (96, 32), (40, 16)])
def test_fused_1_step_vs_reference(reference, nx, ny):
    p, uu = ic.orszag_tang(nx, ny, di=0.05)
    ru, _ = run_ref(reference, p, uu, 1, 1e-3)
    with Domain(p, uu) as d:
        d.steps(1, 1e-3, fused=True)
        err = rel_l2(d.get("uu"), ru)
    assert err.max() < 1e-12, err


def test_fused_multi_step_vs_reference(reference):
    p, uu = ic.orszag_tang(128, 64, di=0.05)
    ru, _ = run_ref(reference, p, uu, 7, 1e-3)
    with Domain(p, uu) as d:
        d.steps(3, 1e-3, fused=True)   # two calls: the pending x filter is
        d.steps(4, 1e-3, fused=True)   # settled at the end of each call
        err = rel_l2(d.get("uu"), ru)
    assert err.max() < 1e-11, err


def test_fused_256_100_steps_vs_reference(reference):
    p, uu = ic.orszag_tang(256, 256, di=0.05)
    ru, _ = run_ref(reference, p, uu, 100, 1e-3)
    with Domain(p, uu) as d:
        d.steps(100, 1e-3, fused=True)
        gu = d.get("uu")
    err = rel_l2(gu, ru)
    assert err.max() < 1e-9, err
    assert O.energy(p, gu) == pytest.approx(O.energy(p, ru), rel=1e-12)
    assert O.cross_helicity(p, gu) == pytest.approx(O.cross_helicity(p, ru), rel=1e-12, abs=1e-14)


@pytest.mark.parametrize("nx,ny", [(4096, 64), (8192, 32), (2048, 128), (1000, 64)])
def test_fused_matches_operator_path_long_lines(nx, ny):
    p, uu = ic.alfvenic_turbulence(nx, ny, mmax=8)
    with Domain(p, uu) as d:
        d.steps(1, 2e-4)
        a = d.get("uu")
        d.set("uu", uu)
        d.steps(1, 2e-4, fused=True)
        b = d.get("uu")
    assert rel_l2(b, a).max() < 1e-12


def test_fused_cfl_and_hyperbolic_cleaning_vs_reference(reference):
    p, uu = ic.orszag_tang(64, 32, di=0.05, divBcleaning=2)
    uu[8] = 1e-3 * np.random.default_rng(7).standard_normal(uu.shape[1:])
    for dt_fixed in (1e-3, -1.0):
        ru, rdt = run_ref(reference, p, uu, 3, dt_fixed)
        with Domain(p, uu) as d:
            dt = d.steps(3, dt_fixed, fused=True)
            err = rel_l2(d.get("uu"), ru)
        assert dt == pytest.approx(rdt, rel=1e-12)
        assert err.max() < 1e-11, err


def test_fused_diffusive_cleaning_routes_to_operator_stage(reference):
    p, uu = ic.orszag_tang(64, 32, di=0.05, divBcleaning=1)
    ru, _ = run_ref(reference, p, uu, 2, 1e-3)
    with Domain(p, uu) as d:
        d.steps(2, 1e-3, fused=True)
        err = rel_l2(d.get("uu"), ru)
    assert err.max() < 1e-11, err


def test_fused_cfl_steps_match_operator_steps():
    # device step control (dt, Ch, Cp on the device, steps replayed as CUDA
    # graphs) against the host-controlled operator path
    p, uu = ic.orszag_tang(128, 64, di=0.05)
    with Domain(p, uu) as a, Domain(p, uu) as b:
        dta = a.steps(6, 0.0, dt=1e-3)
        dtb = b.steps(6, 0.0, dt=1e-3, fused=True)
        assert dtb == pytest.approx(dta, rel=1e-12)
        assert rel_l2(b.get("uu"), a.get("uu")).max() < 1e-11


@pytest.mark.parametrize("dt_fixed", [1e-3, 0.0])
def test_graph_replay_equals_step_by_step(dt_fixed):
    # one call of 6 steps (first eager, then the captured step replayed)
    # against 6 calls of one step (all eager): the same launches, bit for bit
    p, uu = ic.alfvenic_turbulence(256, 128, mmax=8)
    with Domain(p, uu) as a, Domain(p, uu) as b:
        dta = a.steps(6, dt_fixed, dt=2e-4, fused=True)
        dtb = 2e-4
        for _ in range(6):
            dtb = b.steps(1, dt_fixed, dt=dtb, fused=True)
        assert dta == dtb
        np.testing.assert_array_equal(a.get("uu"), b.get("uu"))


def test_hyperbolic_cleaning_fused_fixed_dt_vs_reference(reference):
    p, uu = ic.orszag_tang(64, 64, di=0.05, divBcleaning=2)
    ru, _ = run_ref(reference, p, uu, 5, 1e-3)
    with Domain(p, uu) as d:
        d.steps(5, 1e-3, fused=True)
        err = rel_l2(d.get("uu"), ru)
    assert err.max() < 1e-11, err


@pytest.mark.parametrize("nx,ny", [(4096, 64), (256, 256)])
def test_autotune_keeps_the_results(nx, ny):
    # every tile width solves the same systems exactly: the tuned steps agree
    # with the default ones to rounding
    p, uu = ic.alfvenic_turbulence(nx, ny, mmax=8)
    with Domain(p, uu) as a, Domain(p, uu) as b:
        w = b.autotune()
        assert w in (0, 8, 16, 32)  # 0: the chunked x pass
        a.steps(3, 2e-4, fused=True)
        b.steps(3, 2e-4, fused=True)
        assert rel_l2(b.get("uu"), a.get("uu")).max() < 1e-12


def test_diffusive_cleaning_fused_vs_reference(reference):
    # divBcleaning = 1: the y pass splits around calcDivB and the operator
    # derivatives of divB (mhd.c:175-182)
    p, uu = ic.orszag_tang(64, 64, di=0.05, divBcleaning=1)
    ru, _ = run_ref(reference, p, uu, 5, 1e-3)
    with Domain(p, uu) as d:
        d.steps(5, 1e-3, fused=True)
        err = rel_l2(d.get("uu"), ru)
    assert err.max() < 1e-11, err


def test_diffusive_cleaning_fused_matches_operator_path_long_lines():
    p, uu = ic.orszag_tang(4096, 64, di=0.05, divBcleaning=1)
    with Domain(p, uu) as a, Domain(p, uu) as b:
        a.steps(3, 1e-4)
        b.steps(3, 1e-4, fused=True)
        assert rel_l2(b.get("uu"), a.get("uu")).max() < 1e-12


@pytest.mark.parametrize("mixed", [False, True])
def test_checkpoint_restart_is_exact(tmp_path, mixed):
    # a job paused at a step boundary (state written in the reference's
    # out%04d.dat format, writeOutput.c) and resumed in a new context gives the
    # same fields bit for bit: dudtRK is reset every step, so uu is the state
    from mhd2dcfdfftw_open_b200 import dumpio
    p, uu = ic.alfvenic_turbulence(256, 128, mmax=8)
    with Domain(p, uu) as a:
        a.set_precision(mixed)
        a.steps(10, 2e-4, fused=True)
        full = a.get("uu")
    with Domain(p, uu) as b:
        b.set_precision(mixed)
        b.steps(5, 2e-4, fused=True)
        dumpio.write_state(str(tmp_path / "out0001.dat"), b.get("uu"), 5 * 2e-4)
    t, saved = dumpio.read_state(str(tmp_path / "out0001.dat"), p.nvar, p.nx, p.ny)
    assert t == pytest.approx(1e-3)
    with Domain(p, saved) as c:
        c.set_precision(mixed)
        c.steps(5, 2e-4, fused=True)
        np.testing.assert_array_equal(c.get("uu"), full)
