"""ctypes driver of the reference solver built from its own sources
(oracle/_ref/libmhdref.so, see oracle/Makefile and oracle/ref_harness.c).

TEST INFRASTRUCTURE ONLY: used by tests/ and bench.py's CPU-baseline leg as
the checker, never by the product.

The reference keeps all state in C globals, so one process holds one
configuration at a time; ``Reference.setup`` re-runs ``initialize()`` for a
new configuration (leaking the previous arrays, as the reference has no full
teardown).  Arrays are exchanged as numpy float64 in the reference layout
``[NVAR][nx][ny]``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(REF_DIR, "libmhdref.so")
BIN_PATH = os.path.join(REF_DIR, "mhd_ref")

_dp = ctypes.POINTER(ctypes.c_double)


def available() -> bool:
    return os.path.exists(LIB_PATH) and os.path.exists(BIN_PATH)


def ref_dir() -> str:
    """Where the reference's C sources are: $MHD_REF_DIR, else the default
    of oracle/Makefile (its `REF_DIR ?=` line, the one place that names it)."""
    env = os.environ.get("MHD_REF_DIR")
    if env:
        return env
    with open(os.path.join(HERE, "Makefile")) as f:
        for line in f:
            m = line.split("?=", 1)
            if len(m) == 2 and m[0].strip() == "REF_DIR":
                return m[1].strip()
    return ""


def sources_present() -> bool:
    d = ref_dir()
    return bool(d) and os.path.isfile(os.path.join(d, "calcDerivs.c"))


def build(src_dir: str | None = None) -> None:
    """Compile the reference from its sources (needs the reference tree)."""
    d = src_dir or ref_dir()
    if not d or not os.path.isdir(d):
        raise FileNotFoundError(d or "MHD_REF_DIR")
    subprocess.run(["make", "-s", "-C", HERE, f"REF_DIR={d}"], check=True)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


class Reference:
    def __init__(self):
        if not available():
            raise RuntimeError("reference oracle not built (make -C oracle)")
        self.lib = ctypes.CDLL(LIB_PATH)
        L = self.lib
        L.ref_setup.argtypes = [ctypes.c_char_p]
        L.ref_steps.restype = ctypes.c_double
        L.ref_steps.argtypes = [ctypes.c_int, ctypes.c_double, _dp]
        L.ref_check_divb.restype = ctypes.c_double
        L.ref_stage.argtypes = [ctypes.c_int]
        L.ref_nvar.restype = ctypes.c_long
        for f in ("derivX", "derivXX"):
            getattr(L, f).argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int]
        for f in ("derivY", "derivYY"):
            getattr(L, f).argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_int]
        L.calcDt.restype = ctypes.c_double
        L.calcDt.argtypes = [ctypes.c_double]
        L.rkInit.argtypes = [ctypes.c_double]
        L.rkExecute.argtypes = [ctypes.c_int]
        self.p = None
        self._tmp = tempfile.TemporaryDirectory(prefix="mhdref_")

    # -- globals -----------------------------------------------------------
    def _gptr(self, name):
        return ctypes.c_void_p.in_dll(self.lib, name).value

    def garray(self, name, nfields):
        """numpy view of a global array (nfields x nx x ny)."""
        addr = self._gptr(name)
        n = nfields * self.p.nx * self.p.ny
        buf = (ctypes.c_double * n).from_address(addr)
        return np.ctypeslib.as_array(buf).reshape(nfields, self.p.nx, self.p.ny)

    def gdouble(self, name):
        return ctypes.c_double.in_dll(self.lib, name)

    # -- configuration -----------------------------------------------------
    def setup(self, p):
        self.p = p
        wd = self._tmp.name
        p.write(os.path.join(wd, "input"))
        rc = self.lib.ref_setup(wd.encode())
        if rc != 0:
            raise RuntimeError(f"ref_setup failed ({rc})")
        self.nvar = int(self.lib.ref_nvar())

    @property
    def uu(self):
        return self.garray("uu", self.nvar)

    def set_state(self, uu):
        self.uu[...] = uu

    # -- runs --------------------------------------------------------------
    def steps(self, nsteps, dt_fixed, dt=0.0):
        d = ctypes.c_double(dt)
        sec = self.lib.ref_steps(int(nsteps), float(dt_fixed), ctypes.byref(d))
        return sec, d.value

    def check_divb(self):
        return float(self.lib.ref_check_divb())

    # -- single operators on caller arrays ---------------------------------
    @staticmethod
    def halos(arr):
        """Periodic 2-point halos [nv][2][ny] as parallel.c:13-24 makes them
        at one rank: left = rows nx-2, nx-1; right = rows 0, 1."""
        h0 = np.ascontiguousarray(arr[:, -2:, :])
        h1 = np.ascontiguousarray(arr[:, :2, :])
        return h0, h1

    def deriv_x(self, arr, order=1):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        nv = arr.shape[0]
        h0, h1 = self.halos(arr)
        out = np.zeros_like(arr)
        f = self.lib.derivX if order == 1 else self.lib.derivXX
        f(nv, _ptr(arr), _ptr(h0), _ptr(h1), _ptr(out), 0, 0)
        return out

    def deriv_y(self, arr, order=1):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        out = np.zeros_like(arr)
        f = self.lib.derivY if order == 1 else self.lib.derivYY
        f(arr.shape[0], _ptr(arr), _ptr(out), 0)
        return out

    def filtering(self, uu):
        """filtering() on a state: x then y filter, in place on the global uu
        after a halo exchange (mhd.c:197-198)."""
        self.set_state(uu)
        self.lib.sendrecvHaloPointsX()
        self.lib.filtering()
        return self.uu.copy()

    def calc_dt(self, uu, dt0):
        self.set_state(uu)
        dt = float(self.lib.calcDt(float(dt0)))
        return dt, self.gdouble("Ch_divBcleaning").value, self.gdouble("Cp_divBcleaning").value


def run_binary(p, uu, nsteps, dt, out_path=None, timeout=None):
    """Run oracle/_ref/mhd_ref on (p, uu) for nsteps; returns (json, uu_out)."""
    import json

    from mhd2dcfdfftw_open_b200.dumpio import read_state, write_state

    with tempfile.TemporaryDirectory(prefix="mhdrefbin_") as wd:
        p.write(os.path.join(wd, "input"))
        ic = os.path.join(wd, "ic.dat")
        write_state(ic, uu)
        out = out_path or os.path.join(wd, "out.dat")
        r = subprocess.run([BIN_PATH, wd, ic, str(nsteps), repr(float(dt)), out],
                           capture_output=True, text=True, timeout=timeout, check=True)
        line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
        res = json.loads(line)
        _, u = read_state(out, uu.shape[0], uu.shape[1], uu.shape[2])
        return res, u
