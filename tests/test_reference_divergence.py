"""CPU: drawn serving jobs that leave the finite numbers do so in the
reference's own numerics.

Request 9 of the seeded 100-request serving stream (Orszag-Tang 128^2,
d_i = 0.0933, eta = nu = 1.2185e-4, CFL 0.3 from dt0 = 1e-4) run through the
reference's C code built at one rank turns non-finite between steps 300 and
420 (at the 10-step checkpoint of step 370 when this was written), and a
short job of the same kind (request 8, 213 steps) stays finite.  The GPU
side of the same comparison is tests/test_gpu_long.py.
"""
import numpy as np

from mhd2dcfdfftw_open_b200 import serving


def _first_nonfinite(reference, req, limit):
    p, uu = req.build()
    reference.setup(p)
    reference.set_state(uu)
    dt = req.dt0
    for s in range(10, limit + 1, 10):
        _, dt = reference.steps(10, 0.0, dt)
        if not np.isfinite(reference.uu).all():
            return s
    return None


def test_drawn_ot_job_diverges_in_the_reference(reference):
    reqs = {q.rid: q for q in serving.draw_requests(100)}
    bad = _first_nonfinite(reference, reqs[9], 600)
    assert bad is not None and 300 <= bad <= 420, bad
    assert _first_nonfinite(reference, reqs[8], 210) is None
