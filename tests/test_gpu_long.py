"""GPU: the configurations at their stated lengths, against the reference.

* Orszag-Tang 256^2, fixed dt = 1e-3, 500 RK3 steps (the CPU-runnable
  configuration, d_i in {0, 0.05}), field by field against the reference's
  own C code built at one rank.  Gate: per-field relative L2 (each field
  against its own norm; uz and Bz stay exactly zero) <= 1e-8 after 500 steps
  (1e-9 after 100 steps, 1e-12 after one: test_gpu_steps.py).
* A drawn serving job that leaves the finite numbers (Orszag-Tang 128^2,
  d_i = 0.0933, eta = nu = 1.2185e-4, CFL 0.3, request 9 of the seeded
  100-request stream): the FP64 GPU path and the reference advance in
  lockstep, 10 steps at a time, agree to 1e-12 through step 300 (past the
  step where the pressure turns negative, 237, in both) and to 1e-9 through
  step 350, and turn non-finite (NaN or Inf) within one 10-step checkpoint
  of each other (step 370 in the reference).
* The serving form's precision gate: two jobs served together in mixed
  precision, 1000 steps each, against the same jobs in FP64, per-field
  relative L2 against each field's own norm <= 1e-5.
"""
import numpy as np
import pytest

from conftest import rel_l2_own
from mhd2dcfdfftw_open_b200 import ic, serving
from mhd2dcfdfftw_open_b200.solver import Domain

pytestmark = pytest.mark.gpu

TOL_500 = 1e-8
TOL_MIXED_1000 = 1e-5


@pytest.fixture(scope="module")
def ot256_reference(reference):
    """The reference's state after 100 and 500 steps (fixed dt: d_i does not
    enter, so one run serves both values of d_i)."""
    p, uu = ic.orszag_tang(256, 256, di=0.05)
    reference.setup(p)
    reference.set_state(uu)
    reference.steps(100, 1e-3)
    at100 = reference.uu.copy()
    reference.steps(400, 1e-3)
    return at100, reference.uu.copy()


@pytest.mark.parametrize("di,fused", [(0.0, True), (0.05, True), (0.05, False)])
def test_orszag_tang_256_500_steps_vs_reference(ot256_reference, di, fused):
    at100, at500 = ot256_reference
    p, uu = ic.orszag_tang(256, 256, di=di)
    with Domain(p, uu) as d:
        d.steps(100, 1e-3, fused=fused)
        e100 = rel_l2_own(d.get("uu"), at100)
        d.steps(400, 1e-3, fused=fused)
        e500 = rel_l2_own(d.get("uu"), at500)
    print(f"OT 256^2 d_i={di} {'fused' if fused else 'operators'}: "
          f"max rel L2 {e100.max():.3e} at 100 steps, {e500.max():.3e} at 500 steps")
    assert e100.max() < 1e-9, e100
    assert e500.max() < TOL_500, e500


def _request9():
    r = [q for q in serving.draw_requests(100) if q.rid == 9][0]
    assert r.kind == "ot" and (r.nx, r.ny) == (128, 128)
    return r


def test_diverging_job_matches_reference_until_it_blows_up(reference):
    r = _request9()
    p, uu = r.build()
    reference.setup(p)
    reference.set_state(uu)
    rdt = gdt = r.dt0
    ref_bad = gpu_bad = None
    errs = []
    with Domain(p, uu) as d:
        for s in range(10, 600, 10):
            if ref_bad is None:
                _, rdt = reference.steps(10, 0.0, rdt)
                if not np.isfinite(reference.uu).all():
                    ref_bad = s
            if gpu_bad is None:
                gdt = d.steps(10, 0.0, dt=gdt, fused=True)
                if not np.isfinite(d.get("uu")).all():
                    gpu_bad = s
            if ref_bad is None and gpu_bad is None:
                errs.append((s, float(rel_l2_own(d.get("uu"), reference.uu).max()),
                             abs(gdt - rdt) / rdt))
            if ref_bad is not None and gpu_bad is not None:
                break
    print("non-finite at step", ref_bad, "(reference),", gpu_bad, "(GPU)")
    print("max rel L2 / dt difference:",
          [(s, f"{e:.2e}", f"{t:.1e}") for s, e, t in errs if s % 50 == 0 or s > 250])
    assert ref_bad is not None and 300 <= ref_bad <= 420
    # The pressure turns negative at step 237 in both and both carry on; the
    # fields agree to ~1e-13 through step 300 and ~1e-11 through 350.  In the
    # last steps before the blow-up the scheme amplifies any difference by
    # about 1e4 per 10 steps, so the NaN arrives within one checkpoint.
    assert max(e for s, e, _ in errs if s <= 300) < 1e-12
    assert max(e for s, e, _ in errs if s <= 350) < 1e-9
    assert gpu_bad is not None and abs(gpu_bad - ref_bad) <= 10


def _served(reqs, mixed):
    for q in reqs:
        q.mixed = mixed
        q.keep_state = True
    res, _ = serving.run_stream(reqs, slots=len(reqs), realtime=False)
    assert all(x.error is None for x in res), [x.error for x in res]
    return {x.rid: x.uu for x in res}


def test_mixed_serving_field_error_after_1000_steps():
    def reqs():
        return [serving.Request(0, 256, 256, 1000, di=0.05, eta=1e-4, nu=1e-4, kind="ot",
                                dt_fixed=1e-3),
                serving.Request(1, 128, 128, 1000, di=0.03, eta=3e-4, nu=3e-4,
                                kind="turbulence", seed=11)]
    mixed = _served(reqs(), True)
    fp64 = _served(reqs(), False)
    for rid in (0, 1):
        err = rel_l2_own(mixed[rid], fp64[rid])
        print(f"job {rid}: per-field relative L2 (own norm) after 1000 steps", np.array2string(err, precision=2))
        assert err.max() < TOL_MIXED_1000, err


@pytest.mark.parametrize("path", ["operators", "fused", "mixed"])
@pytest.mark.parametrize("nx,ny", [(64, 64), (64, 4096)])
def test_out_of_plane_fields_of_a_2d_flow_stay_exactly_zero(path, nx, ny):
    """uz and Bz of the Orszag-Tang vortex are zero and have no source; the
    reference's per-field real transforms keep them exactly zero, and so
    must every GPU path (no rounding leaking in from a packed partner; rows
    of 4096 points take the real-row transforms of Ex and Ez)."""
    p, uu = ic.orszag_tang(nx, ny, di=0.05)
    with Domain(p, uu) as d:
        if path == "mixed":
            d.set_precision(True)
        d.steps(30, 0.0, dt=1e-4, fused=path != "operators")
        out = d.get("uu")
    assert not out[3].any() and not out[6].any()
