"""CPU: host logic -- the `input` layout, dump format, initial conditions and
the C-ABI library's exported symbols (no compute calls without a GPU)."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from mhd2dcfdfftw_open_b200 import dumpio, ic
from mhd2dcfdfftw_open_b200.config import InputParams


def test_input_roundtrip_keeps_16_characters(tmp_path):
    p = InputParams(nx=4096, ny=2048, Lx=2 * math.pi, Ly=20 * math.pi, di=0.05)
    path = tmp_path / "input"
    p.write(str(path))
    lines = path.read_text().splitlines()
    assert len(lines) == 15
    q = InputParams.read(str(path))
    assert q.nx == 4096 and q.ny == 2048
    # 2*pi does not fit in 16 characters: the parsed value is the truncation
    assert q.Lx == float(lines[6][:16])
    assert abs(q.Lx - 2 * math.pi) < 1e-13


def test_reads_reference_style_input(tmp_path):
    text = ("1                   ; boundary condition along x. 0: periodic, 1: open\n"
            "0.5                 ; cfl\n10                  ; Tmax\n0.1                 ; dtOut\n"
            "512                 ; nx\n256                 ; ny \n2.0                 ; Lx\n"
            "4.0                 ; Ly\n1.666666667         ; adiabatic_index\n"
            "0                   ; Hall effect 0: off; 1: on\n0.002               ; di\n"
            "1e-4                ; resistivity\n0                   ; viscosity\n"
            "0                   ; divB cleaning\n1                   ; output divB\n")
    path = tmp_path / "input"
    path.write_text(text)
    q = InputParams.read(str(path))
    assert (q.boundaryTypeX, q.nx, q.ny, q.Hall, q.outDivB) == (1, 512, 256, 0, 1)
    assert q.resistivity == 1e-4 and q.adiabaticIdx == 1.666666667
    assert q.nvar == 8 and q.dx == 2.0 / 511


def test_c_reader_matches_python_reader(tmp_path):
    lib_path = os.path.join(ROOT, "mhd2dcfdfftw_open_b200", "libmhdgpu.so")
    if not os.path.exists(lib_path):
        pytest.skip("libmhdgpu.so not built")
    from mhd2dcfdfftw_open_b200.config import CParams
    from mhd2dcfdfftw_open_b200.solver import load_library
    L = load_library()
    p = InputParams(nx=100, ny=64, Lx=20 * math.pi, di=0.1, divBcleaning=2, Hall=1)
    path = tmp_path / "input"
    p.write(str(path))
    cp = CParams()
    assert L.mhdgpu_read_input(str(path).encode(), ctypes.byref(cp)) == 0
    q = InputParams.read(str(path))
    for name, _ in CParams._fields_:
        assert getattr(cp, name) == getattr(q, name), name


def test_dump_roundtrip(tmp_path):
    uu = np.random.default_rng(0).standard_normal((8, 6, 4))
    dumpio.write_state(str(tmp_path / "out0000.dat"), uu, 1.5)
    t, back = dumpio.read_state(str(tmp_path / "out0000.dat"), 8, 6, 4)
    assert t == 1.5 and np.array_equal(back, uu)
    g = np.arange(6) * 0.5
    dumpio.write_grid(str(tmp_path / "xgrid.dat"), g)
    assert np.array_equal(dumpio.read_grid(str(tmp_path / "xgrid.dat")), g)


def test_initial_conditions():
    p, uu = ic.orszag_tang(32, 16)
    assert uu.shape == (8, 32, 16) and np.allclose(uu[0], (5 / 3) ** 2)
    p, uu = ic.alfvenic_turbulence(64, 64, mmax=8)
    db = uu[4:7] - np.array([1.0, 0, 0])[:, None, None]
    assert math.sqrt(float(np.mean(np.sum(db ** 2, axis=0)))) == pytest.approx(0.5, rel=1e-12)
    assert np.allclose(uu[1:4], db)  # dv = dB
    # divergence free: spectral divergence of dB vanishes
    kx = np.fft.fftfreq(64, d=p.dx) * 2 * np.pi
    ky = np.fft.fftfreq(64, d=p.dy) * 2 * np.pi
    div = np.fft.ifft2(1j * kx[:, None] * np.fft.fft2(db[0]) + 1j * ky[None, :] * np.fft.fft2(db[1]))
    assert np.abs(div).max() < 1e-12
    p, uu = ic.parametric_decay(64, 16)
    assert np.abs(uu[0] - 1).max() <= 1e-3 and np.allclose(uu[5] ** 2 + uu[6] ** 2, 0.04)
    jobs = ic.ensemble_jobs()
    assert len(jobs) == 64 and jobs == ic.ensemble_jobs()
    reqs = ic.serving_requests(n=50)
    assert all(b.arrival > a.arrival for a, b in zip(reqs, reqs[1:]))


def _declared_functions(headers=("mhd_gpu.h",)):
    """Functions declared in the C-ABI headers (mhd_gpu.h: libmhdgpu.so;
    mhd_gpu_dropin.h: the drop-in archive, checked below)."""
    names = []
    for h in headers:
        path = os.path.join(ROOT, "include", h)
        if not os.path.exists(path):
            continue
        text = re.sub(r"/\*.*?\*/", "", open(path).read(), flags=re.S)
        names += re.findall(r"\b(\w+)\s*\([^;{]*\)\s*;", text)
    return [n for n in names if n not in ("if", "while")]


def test_library_exports_every_declared_symbol():
    lib_path = os.path.join(ROOT, "mhd2dcfdfftw_open_b200", "libmhdgpu.so")
    if not os.path.exists(lib_path):
        pytest.skip("libmhdgpu.so not built")
    lib = ctypes.CDLL(lib_path)
    declared = [n for n in _declared_functions() if n.startswith("mhdgpu_")]
    assert len(declared) >= 25
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing


def test_dropin_archive_defines_the_reference_entry_points():
    import subprocess
    arc = os.path.join(ROOT, "mhd2dcfdfftw_open_b200", "libmhdgpu_dropin.a")
    if not os.path.exists(arc):
        pytest.skip("libmhdgpu_dropin.a not built")
    text = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "mhd_gpu_dropin.h")).read(),
                  flags=re.S)
    declared = set(re.findall(r"\b(\w+)\s*\([^;{]*\)\s*;", text))
    out = subprocess.run(["nm", arc], capture_output=True, text=True, check=True).stdout
    defined = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert declared and declared <= defined, declared - defined
