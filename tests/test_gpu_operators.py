"""GPU parity of every hot-path operator against the oracle (and the
reference itself where it is built), through the C ABI.

Tolerances: the finite-difference operators agree with the reference to
rounding (1e-13 relative per field is asserted); spectral operators differ
from FFTW/numpy by the FFT's own rounding (1e-13 relative).
"""
import numpy as np
import pytest

import mhd_oracle as O
from conftest import rel_l2
from mhd2dcfdfftw_open_b200 import ic
from mhd2dcfdfftw_open_b200.solver import Domain

pytestmark = pytest.mark.gpu

SIZES = [(16, 16), (64, 32), (40, 8), (256, 64), (1024, 32), (4096, 64), (8192, 32)]
TOL = 1e-13


def rand_state(p, seed=0):
    rng = np.random.default_rng(seed)
    uu = rng.standard_normal(p.state_shape())
    uu[0] = 1.5 + 0.3 * np.abs(uu[0])
    uu[7] = 1.0 + 0.3 * np.abs(uu[7])
    return uu


@pytest.mark.parametrize("nx,ny", SIZES)
def test_derivx_all_orders(nx, ny):
    p, _ = ic.orszag_tang(nx, ny)
    uu = rand_state(p)
    with Domain(p, uu) as d:
        d.derivX(p.nvar)
        assert rel_l2(d.get("dudx"), O.derivX(uu, p.dx)).max() < TOL
        d.derivXX(3, "uu", 1, "d2udx2")
        assert rel_l2(d.get("d2udx2"), O.derivXX(uu[1:4], p.dx)).max() < TOL
        d.derivXX(3, "uu", 4, "d2Bdx2")
        assert rel_l2(d.get("d2Bdx2"), O.derivXX(uu[4:7], p.dx)).max() < TOL


@pytest.mark.parametrize("nx,ny", SIZES)
def test_derivy_all_orders(nx, ny):
    p, _ = ic.orszag_tang(nx, ny)
    uu = rand_state(p, 1)
    with Domain(p, uu) as d:
        d.derivY(p.nvar)
        assert rel_l2(d.get("dudy"), O.derivY(uu, p.Ly)).max() < TOL
        d.derivYY(3, "uu", 1, "d2udy2")
        assert rel_l2(d.get("d2udy2"), O.derivYY(uu[1:4], p.Ly)).max() < TOL


@pytest.mark.parametrize("nx,ny", SIZES)
def test_filtering(nx, ny):
    p, _ = ic.orszag_tang(nx, ny)
    uu = rand_state(p, 2)
    with Domain(p, uu) as d:
        d.filtering()
        assert rel_l2(d.get("uu"), O.filtering(uu)).max() < TOL


def test_efield_rhs_rk():
    p, uu = ic.orszag_tang(64, 32, di=0.05)
    uu = uu + 0.01 * rand_state(p, 3)
    with Domain(p, uu) as d:
        d.calcEfield()
        E = O.calcEfield(uu)
        assert rel_l2(d.get("Efield"), E).max() < 1e-15
        for name, arr in (("dudx", O.derivX(uu, p.dx)), ("dudy", O.derivY(uu, p.Ly))):
            d.set(name, arr)
        d.derivXX(3, "uu", 1, "d2udx2")
        d.derivYY(3, "uu", 1, "d2udy2")
        d.derivXX(3, "uu", 4, "d2Bdx2")
        d.derivYY(3, "uu", 4, "d2Bdy2")
        d.derivX(3, "Efield", 0, "dEdx")
        d.derivY(3, "Efield", 0, "dEdy")
        d.calcRHS()
        ref = O.calcRHS(p, uu, O.derivX(uu, p.dx), O.derivY(uu, p.Ly), O.derivX(E, p.dx),
                        O.derivY(E, p.Ly), O.derivXX(uu[1:4], p.dx), O.derivYY(uu[1:4], p.Ly),
                        O.derivXX(uu[4:7], p.dx), O.derivYY(uu[4:7], p.Ly))
        dudt = d.get("dudt")
        assert rel_l2(dudt, ref).max() < 1e-12
        d.rkInit(1e-3)
        d.rkExecute(0)
        u1, r1 = O.rkExecute(uu, dudt, np.zeros_like(uu), 0, 1e-3)
        assert rel_l2(d.get("uu"), u1).max() < 1e-15
        assert np.array_equal(d.get("dudtRK"), r1)


@pytest.mark.parametrize("cleaning", [0, 2])
def test_calc_dt(cleaning):
    p, uu = ic.orszag_tang(64, 32, di=0.05, divBcleaning=cleaning)
    if cleaning == 2:
        uu[8] = 0.01 * rand_state(p, 4)[1]
    with Domain(p, uu) as d:
        for dt0 in (0.0, 1e-3):
            dt = d.calcDt(dt0)
            dto, Ch, Cp = O.calcDt(p, uu, dt0)
            assert dt == pytest.approx(dto, rel=1e-14)
            if cleaning == 2:
                ch, cp = d.cleaning_speeds()
                assert ch == pytest.approx(Ch, rel=1e-14)
                assert cp == pytest.approx(Cp, rel=1e-14)


def test_derivx_against_reference(reference):
    p, _ = ic.orszag_tang(64, 32)
    uu = rand_state(p, 5)
    reference.setup(p)
    with Domain(p, uu) as d:
        d.derivX(p.nvar)
        assert rel_l2(d.get("dudx"), reference.deriv_x(uu, 1)).max() < TOL
        d.derivY(p.nvar)
        assert rel_l2(d.get("dudy"), reference.deriv_y(uu, 1)).max() < TOL
