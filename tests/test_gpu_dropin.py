"""GPU: the drop-in layer under the reference's own driver.

oracle/_ref/mhd_refmain is the reference's mhd.c + usrInitialize.c linked with
the reference's numerics; oracle/_ref/mhd_dropin is the same driver linked with
libmhdgpu_dropin.a in place of calcDerivs/calcRHS/filtering/timeAdvance/
parallel (oracle/Makefile, target `dropin`).  Both run the same `input` with
the reference's CFL control and output cadence; every dump they write must
agree (per-field relative L2, 1e-10 after a few RK3 steps of the reference's
current-sheet initial condition).
"""
import glob
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_l2
from mhd2dcfdfftw_open_b200.config import InputParams
from mhd2dcfdfftw_open_b200.dumpio import read_state

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref")


def run(exe, wd, p, env=None):
    os.makedirs(wd, exist_ok=True)
    p.write(os.path.join(wd, "input"))
    r = subprocess.run([exe], cwd=wd, capture_output=True, text=True, timeout=300,
                       env=None if env is None else {**os.environ, **env})
    assert r.returncode == 0, r.stderr[-2000:]
    assert "drop-in" not in r.stderr, r.stderr
    return sorted(os.path.basename(f) for f in glob.glob(os.path.join(wd, "*.dat")))


@pytest.mark.parametrize("resident", [False, True])
@pytest.mark.parametrize("nx,ny,cleaning", [(64, 32, 0), (48, 64, 2)])
def test_reference_driver_with_dropin_matches_reference(tmp_path, nx, ny, cleaning, resident):
    """resident: the driver with the sync hook before each checkDivB
    (oracle/_ref/mhd_dropin_resident), arrays kept on the device between
    calls (MHDGPU_DROPIN_RESIDENT=1)."""
    gpu = "mhd_dropin_resident" if resident else "mhd_dropin"
    exes = [os.path.join(REF, "mhd_refmain"), os.path.join(REF, gpu)]
    if not all(os.path.exists(e) for e in exes):
        pytest.skip("drop-in demo not built (make -C oracle dropin)")
    p = InputParams(boundaryTypeX=0, cfl=0.3, Tmax=0.02, dtOut=0.01, nx=nx, ny=ny, Lx=2.0,
                    Ly=4.0, adiabaticIdx=5 / 3, Hall=1, di=0.05, resistivity=1e-3,
                    viscosity=1e-3, divBcleaning=cleaning, outDivB=1)
    fa = run(exes[0], str(tmp_path / "ref"), p)
    fb = run(exes[1], str(tmp_path / "gpu"), p,
             env={"MHDGPU_DROPIN_RESIDENT": "1"} if resident else None)
    assert fa == fb and "out0002.dat" in fa
    nvar = p.nvar
    for name in fa:
        if name.startswith("out"):
            ta, a = read_state(str(tmp_path / "ref" / name), nvar, nx, ny)
            tb, b = read_state(str(tmp_path / "gpu" / name), nvar, nx, ny)
            assert ta == pytest.approx(tb, rel=1e-12)
            assert rel_l2(b, a).max() < 1e-10, name
        elif name.startswith("divB"):
            a = np.fromfile(str(tmp_path / "ref" / name))[1:]
            b = np.fromfile(str(tmp_path / "gpu" / name))[1:]
            assert np.abs(a - b).max() <= 1e-9 * max(1.0, np.abs(a).max()), name
