"""Host-side mirror of the reference's hot-path interface over the C ABI.

``Domain`` owns one GPU context (``include/mhd_gpu.h``) and exposes the
reference's operators under the reference's names -- ``derivX``, ``derivXX``,
``derivY``, ``derivYY`` (calcDerivs.c), ``calcEfield``, ``calcDivB``,
``calcRHS`` (calcRHS.c), ``filtering`` (filtering.c), ``rkInit``,
``rkExecute``, ``calcDt`` (timeAdvance.c) and ``checkDivB`` (mhd.c) -- acting
on the context's device arrays, which mirror the reference's globals
(``uu``, ``dudx``, ``dudy``, ``d2udx2``, ...).  Arrays cross the boundary as
numpy float64 in the reference layout ``[nfield][nx][ny]``.

The shared library is required: importing works without it, but every call
raises ``RuntimeError`` when ``libmhdgpu.so`` is missing or no GPU is present.
There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .config import CParams, InputParams

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmhdgpu.so")

# mhdgpu_array (include/mhd_gpu.h)
UU, DUDX, DUDY, D2UDX2, D2UDY2, D2BDX2, D2BDY2, DIVB, DDIVBDX, DDIVBDY, \
    EFIELD, DEDX, DEDY, DUDT, DUDTRK = range(15)
ARRAY_NAMES = {
    "uu": UU, "dudx": DUDX, "dudy": DUDY, "d2udx2": D2UDX2, "d2udy2": D2UDY2,
    "d2Bdx2": D2BDX2, "d2Bdy2": D2BDY2, "divB": DIVB, "ddivBdx": DDIVBDX,
    "ddivBdy": DDIVBDY, "Efield": EFIELD, "dEdx": DEDX, "dEdy": DEDY,
    "dudt": DUDT, "dudtRK": DUDTRK,
}

EXPORTED = (
    "mhdgpu_read_input", "mhdgpu_create", "mhdgpu_destroy", "mhdgpu_last_error",
    "mhdgpu_error_string", "mhdgpu_nvar", "mhdgpu_set_array", "mhdgpu_get_array",
    "mhdgpu_device_array", "mhdgpu_synchronize", "mhdgpu_deriv_x", "mhdgpu_deriv_y",
    "mhdgpu_calc_efield", "mhdgpu_calc_divb", "mhdgpu_calc_rhs", "mhdgpu_rk_init",
    "mhdgpu_rk_execute", "mhdgpu_filtering", "mhdgpu_calc_dt", "mhdgpu_check_divb",
    "mhdgpu_get_cleaning_speeds", "mhdgpu_stage", "mhdgpu_steps", "mhdgpu_steps_fused",
    "mhdgpu_steps_fused_stream",
    "mhdgpu_diagnostics", "mhdgpu_state_cells", "mhdgpu_stream", "mhdgpu_launch_count", "mhdgpu_profile",
    "mhdgpu_profile_read", "mhdgpu_set_precision", "mhdgpu_autotune", "mhdgpu_selftest_wait",
)

# arithmetic of the fused steps (mhdgpu_set_precision)
PRECISION_FP64 = 0
PRECISION_MIXED = 1

# kernel classes of mhdgpu_profile_read
KCLASSES = ("xsolve", "yspec", "pointwise", "reduce", "fused_x", "fused_y", "fused_xf")

_lib = None


class MhdGpuError(RuntimeError):
    pass


def load_library(path: str = LIB_PATH):
    """Load libmhdgpu.so (no GPU needed to load it)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with "
                           "`python -m mhd2dcfdfftw_open_b200.build`")
    L = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    vp = ctypes.c_void_p
    L.mhdgpu_read_input.argtypes = [ctypes.c_char_p, ctypes.POINTER(CParams)]
    L.mhdgpu_create.argtypes = [ctypes.POINTER(CParams), ctypes.c_int, ctypes.POINTER(vp)]
    L.mhdgpu_destroy.argtypes = [vp]
    L.mhdgpu_destroy.restype = None
    L.mhdgpu_error_string.restype = ctypes.c_char_p
    L.mhdgpu_nvar.argtypes = [vp]
    L.mhdgpu_set_array.argtypes = [vp, ctypes.c_int, dp]
    L.mhdgpu_get_array.argtypes = [vp, ctypes.c_int, dp]
    L.mhdgpu_device_array.argtypes = [vp, ctypes.c_int]
    L.mhdgpu_device_array.restype = vp
    L.mhdgpu_synchronize.argtypes = [vp]
    for f in ("mhdgpu_deriv_x", "mhdgpu_deriv_y"):
        getattr(L, f).argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    for f in ("mhdgpu_calc_efield", "mhdgpu_calc_divb", "mhdgpu_calc_rhs", "mhdgpu_filtering"):
        getattr(L, f).argtypes = [vp]
    L.mhdgpu_rk_init.argtypes = [vp, ctypes.c_double]
    L.mhdgpu_rk_execute.argtypes = [vp, ctypes.c_int]
    L.mhdgpu_calc_dt.argtypes = [vp, ctypes.c_double, dp]
    L.mhdgpu_check_divb.argtypes = [vp, dp]
    L.mhdgpu_get_cleaning_speeds.argtypes = [vp, dp, dp]
    L.mhdgpu_stage.argtypes = [vp, ctypes.c_int]
    L.mhdgpu_steps.argtypes = [vp, ctypes.c_int, ctypes.c_double, dp]
    L.mhdgpu_steps_fused.argtypes = [vp, ctypes.c_int, ctypes.c_double, dp]
    L.mhdgpu_steps_fused_stream.argtypes = [vp, ctypes.c_int, ctypes.POINTER(dp), ctypes.POINTER(dp),
                                            ctypes.c_int, ctypes.c_double, dp]
    L.mhdgpu_set_precision.argtypes = [vp, ctypes.c_int]
    L.mhdgpu_autotune.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.mhdgpu_selftest_wait.argtypes = [vp, ctypes.c_double]
    L.mhdgpu_diagnostics.argtypes = [vp, dp, dp, ctypes.POINTER(ctypes.c_int)]
    L.mhdgpu_state_cells.argtypes = [vp, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_long)]
    L.mhdgpu_stream.argtypes = [vp]
    L.mhdgpu_stream.restype = vp
    L.mhdgpu_launch_count.argtypes = [vp]
    L.mhdgpu_launch_count.restype = ctypes.c_long
    L.mhdgpu_profile.argtypes = [vp, ctypes.c_int]
    L.mhdgpu_profile_read.argtypes = [vp, ctypes.c_int, dp, ctypes.POINTER(ctypes.c_long), dp]
    _lib = L
    return L


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Domain:
    """One periodic 2-D domain resident on one GPU."""

    def __init__(self, params: InputParams, uu: np.ndarray | None = None, device: int = 0):
        self.lib = load_library()
        self.p = params
        cp = CParams.from_params(params)
        h = ctypes.c_void_p()
        self._check(self.lib.mhdgpu_create(ctypes.byref(cp), int(device), ctypes.byref(h)))
        self.h = h
        self.nvar = int(self.lib.mhdgpu_nvar(self.h))
        self.shape = (self.nvar, params.nx, params.ny)
        if uu is not None:
            self.set("uu", uu)

    def _check(self, rc):
        if rc != 0:
            msg = self.lib.mhdgpu_error_string(rc).decode()
            raise MhdGpuError(f"mhdgpu status {rc}: {msg}")
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.lib.mhdgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- arrays ------------------------------------------------------------
    def _nfields(self, which):
        return {UU: self.nvar, DUDX: self.nvar, DUDY: self.nvar, DUDT: self.nvar,
                DUDTRK: self.nvar, DIVB: 1, DDIVBDX: 1, DDIVBDY: 1}.get(which, 3)

    def set(self, name, arr):
        which = ARRAY_NAMES[name]
        n = self._nfields(which)
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(n, self.p.nx, self.p.ny)
        self._check(self.lib.mhdgpu_set_array(self.h, which, _dptr(a)))

    def get(self, name, out=None):
        which = ARRAY_NAMES[name]
        shape = (self._nfields(which), self.p.nx, self.p.ny)
        a = np.empty(shape) if out is None else out
        if a.shape != shape or a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape %s" % (shape,))
        self._check(self.lib.mhdgpu_get_array(self.h, which, _dptr(a)))
        return a

    def device_ptr(self, name):
        return int(self.lib.mhdgpu_device_array(self.h, ARRAY_NAMES[name]))

    def synchronize(self):
        self._check(self.lib.mhdgpu_synchronize(self.h))

    # -- operators, named as in the reference -----------------------------
    def derivX(self, nv, src="uu", start=0, dst="dudx"):
        self._check(self.lib.mhdgpu_deriv_x(self.h, nv, ARRAY_NAMES[src], start, ARRAY_NAMES[dst], 1))

    def derivXX(self, nv, src="uu", start=0, dst="d2udx2"):
        self._check(self.lib.mhdgpu_deriv_x(self.h, nv, ARRAY_NAMES[src], start, ARRAY_NAMES[dst], 2))

    def derivY(self, nv, src="uu", start=0, dst="dudy"):
        self._check(self.lib.mhdgpu_deriv_y(self.h, nv, ARRAY_NAMES[src], start, ARRAY_NAMES[dst], 1))

    def derivYY(self, nv, src="uu", start=0, dst="d2udy2"):
        self._check(self.lib.mhdgpu_deriv_y(self.h, nv, ARRAY_NAMES[src], start, ARRAY_NAMES[dst], 2))

    def calcEfield(self):
        self._check(self.lib.mhdgpu_calc_efield(self.h))

    def calcDivB(self):
        self._check(self.lib.mhdgpu_calc_divb(self.h))

    def calcRHS(self):
        self._check(self.lib.mhdgpu_calc_rhs(self.h))

    def rkInit(self, dt):
        self._check(self.lib.mhdgpu_rk_init(self.h, float(dt)))

    def rkExecute(self, iRK):
        self._check(self.lib.mhdgpu_rk_execute(self.h, int(iRK)))

    def filtering(self):
        self._check(self.lib.mhdgpu_filtering(self.h))

    def calcDt(self, dt0):
        d = ctypes.c_double()
        self._check(self.lib.mhdgpu_calc_dt(self.h, float(dt0), ctypes.byref(d)))
        return d.value

    def checkDivB(self):
        d = ctypes.c_double()
        self._check(self.lib.mhdgpu_check_divb(self.h, ctypes.byref(d)))
        return d.value

    def cleaning_speeds(self):
        ch, cp = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mhdgpu_get_cleaning_speeds(self.h, ctypes.byref(ch), ctypes.byref(cp)))
        return ch.value, cp.value

    # -- stages and steps --------------------------------------------------
    def stage(self, iRK):
        self._check(self.lib.mhdgpu_stage(self.h, int(iRK)))

    def steps(self, nsteps, dt_fixed, dt=0.0, fused=False):
        d = ctypes.c_double(dt)
        f = self.lib.mhdgpu_steps_fused if fused else self.lib.mhdgpu_steps
        self._check(f(self.h, int(nsteps), float(dt_fixed), ctypes.byref(d)))
        return d.value

    def steps_stream(self, inputs, outputs, nsteps, dt_fixed, dt=0.0):
        """Advance each state of `inputs` (arrays shaped like uu) by nsteps
        fused steps from dt, independently, into the matching array of
        `outputs` (C-contiguous float64, preferably page-locked); transfers
        overlap the steps of the neighbouring states.  Returns the last
        state's dt (mhdgpu_steps_fused_stream)."""
        if len(inputs) != len(outputs):
            raise ValueError("inputs and outputs differ in length")
        shape = (self.nvar, self.p.nx, self.p.ny)
        for a in list(inputs) + list(outputs):
            if a.shape != shape or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("states must be C-contiguous float64 arrays of shape %s" % (shape,))
        n = len(inputs)
        dp = ctypes.POINTER(ctypes.c_double)
        pin = (dp * n)(*[_dptr(a) for a in inputs])
        pout = (dp * n)(*[_dptr(a) for a in outputs])
        d = ctypes.c_double(dt)
        self._check(self.lib.mhdgpu_steps_fused_stream(self.h, n, pin, pout, int(nsteps),
                                                       float(dt_fixed), ctypes.byref(d)))
        return d.value

    def set_precision(self, mixed):
        """Arithmetic of the fused steps: FP64 (False, the default) or mixed
        precision (True: FP32 sweeps, butterflies and fluxes, FP64 state and
        RK3 accumulation)."""
        self._check(self.lib.mhdgpu_set_precision(
            self.h, PRECISION_MIXED if mixed else PRECISION_FP64))

    def autotune(self):
        """Pick the fastest tile width of the fused x pass for this grid and
        precision (remembered for later domains of the same shape); returns
        the width, 0 for the chunked x pass of lines of 1024 rows and more."""
        w = ctypes.c_int(0)
        self._check(self.lib.mhdgpu_autotune(self.h, ctypes.byref(w)))
        return w.value

    def diagnostics(self):
        e, h, fin = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self._check(self.lib.mhdgpu_diagnostics(self.h, ctypes.byref(e), ctypes.byref(h),
                                                ctypes.byref(fin)))
        nf, npos = ctypes.c_long(), ctypes.c_long()
        self._check(self.lib.mhdgpu_state_cells(self.h, ctypes.byref(nf), ctypes.byref(npos)))
        return {"energy": e.value, "cross_helicity": h.value, "finite": bool(fin.value),
                "nonfinite_cells": nf.value, "nonpositive_cells": npos.value,
                "positive": nf.value == 0 and npos.value == 0}

    @property
    def uu(self):
        return self.get("uu")

    # -- instrumentation ---------------------------------------------------
    def stream_handle(self) -> int:
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return int(self.lib.mhdgpu_stream(self.h) or 0)

    def launch_count(self) -> int:
        return int(self.lib.mhdgpu_launch_count(self.h))

    def profile(self, enable: bool):
        self._check(self.lib.mhdgpu_profile(self.h, 1 if enable else 0))

    def profile_read(self):
        """{kernel class: (total ms, launches, algorithmic bytes)} of the
        profiled launches."""
        out = {}
        for k, name in enumerate(KCLASSES):
            ms, n, b = ctypes.c_double(), ctypes.c_long(), ctypes.c_double()
            self._check(self.lib.mhdgpu_profile_read(self.h, k, ctypes.byref(ms), ctypes.byref(n),
                                                     ctypes.byref(b)))
            out[name] = (ms.value, n.value, b.value)
        return out
