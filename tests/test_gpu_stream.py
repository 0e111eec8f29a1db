"""GPU: mhdgpu_steps_fused_stream, a stream of independent states through one
context with the transfers overlapping the steps.

Each state of the stream must come out bit for bit as mhdgpu_set_array +
mhdgpu_steps_fused + mhdgpu_get_array give it one at a time, in FP64 and
mixed precision, with fixed dt and CFL control, through the chunked x pass
and the cluster x pass; the context then holds the last state; the dt
returned is the last state's; invalid arguments are refused.
"""
import ctypes
import os

import numpy as np
import pytest
import torch

from mhd2dcfdfftw_open_b200 import ic
from mhd2dcfdfftw_open_b200.solver import Domain

pytestmark = pytest.mark.gpu


def _states(nx, ny, n):
    out = []
    for s in range(n):
        p, uu = ic.alfvenic_turbulence(nx, ny, seed=s + 1, mmax=8)
        out.append(uu)
    return p, out


def _one_at_a_time(p, states, nsteps, dt_fixed, mixed):
    res, dts = [], []
    with Domain(p, states[0]) as d:
        if mixed:
            d.set_precision(True)
        for uu in states:
            d.set("uu", uu)
            dts.append(d.steps(nsteps, dt_fixed, dt=1e-4, fused=True))
            res.append(d.get("uu"))
    return res, dts


@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("cfl", [False, True])
@pytest.mark.parametrize("nx,ny,chunked", [(1024, 64, True), (128, 128, False)])
def test_stream_equals_one_at_a_time(nx, ny, chunked, cfl, mixed):
    saved = os.environ.get("MHDGPU_XN_MIN_NX")
    if not chunked:
        os.environ["MHDGPU_XN_MIN_NX"] = "100000"
    try:
        p, states = _states(nx, ny, 3)
        dtf = 0.0 if cfl else 2e-4
        ref, dts = _one_at_a_time(p, states, 2, dtf, mixed)
        ins = [torch.from_numpy(np.ascontiguousarray(u)).pin_memory().numpy() for u in states]
        outs = [torch.empty(u.shape, dtype=torch.float64).pin_memory().numpy() for u in states]
        with Domain(p, states[0]) as d:
            if mixed:
                d.set_precision(True)
            dt = d.steps_stream(ins, outs, 2, dtf, dt=1e-4)
            last = d.get("uu")
        for a, b in zip(outs, ref):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(last, ref[-1])
        assert dt == dts[-1]
    finally:
        if saved is None:
            os.environ.pop("MHDGPU_XN_MIN_NX", None)
        else:
            os.environ["MHDGPU_XN_MIN_NX"] = saved


def test_stream_with_repeated_pointers_and_pageable_memory():
    p, states = _states(256, 64, 1)
    ref, _ = _one_at_a_time(p, states, 1, 2e-4, False)
    out = np.empty_like(states[0])
    with Domain(p, states[0]) as d:
        d.steps_stream([states[0]] * 4, [out] * 4, 1, 2e-4)
    np.testing.assert_array_equal(out, ref[0])


def test_stream_refuses_invalid_arguments():
    p, states = _states(128, 64, 1)
    with Domain(p, states[0]) as d:
        with pytest.raises(ValueError):
            d.steps_stream([states[0]], [], 1, 2e-4)
        dp = ctypes.POINTER(ctypes.c_double)
        null = (dp * 1)()
        dt = ctypes.c_double(0.0)
        rc = d.lib.mhdgpu_steps_fused_stream(d.h, 1, null, null, 1, 2e-4, ctypes.byref(dt))
        assert rc != 0
        rc = d.lib.mhdgpu_steps_fused_stream(d.h, -1, null, null, 1, 2e-4, ctypes.byref(dt))
        assert rc != 0
        assert d.lib.mhdgpu_steps_fused_stream(d.h, 0, None, None, 1, 2e-4, ctypes.byref(dt)) == 0
