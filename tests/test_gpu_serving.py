"""GPU: jobs served together return the same fields as the same jobs run
alone, one at a time (each job's arithmetic is independent of the others
and deterministic), in FP64 and in mixed precision; the server admits jobs
while others run."""
import numpy as np
import pytest

from mhd2dcfdfftw_open_b200 import serving as S

pytestmark = pytest.mark.gpu


def _jobs(mixed):
    sizes = [(128, 128), (256, 128), (256, 256), (512, 256), (128, 512), (1024, 64)]
    out = []
    for i, (nx, ny) in enumerate(sizes):
        out.append(S.Request(i, nx, ny, steps=40 + 10 * i, di=0.02 * i, eta=2e-4, nu=3e-4,
                             kind="ot" if i % 2 == 0 else "turbulence", seed=11 + i,
                             mixed=mixed, keep_state=True))
    return out


@pytest.mark.parametrize("mixed", [False, True])
def test_same_alone_and_in_the_mix(mixed):
    alone, _ = S.run_stream(_jobs(mixed), slots=1, realtime=False)
    mix, _ = S.run_stream(_jobs(mixed), slots=6, realtime=False)
    assert all(r.error is None for r in alone + mix), [r.error for r in alone + mix]
    for a, b in zip(alone, mix):
        assert a.rid == b.rid
        assert a.dt == b.dt
        np.testing.assert_array_equal(a.uu, b.uu)


def test_mixed_serving_matches_fp64_within_tolerance():
    fp, _ = S.run_stream(_jobs(False), slots=6, realtime=False)
    mx, _ = S.run_stream(_jobs(True), slots=6, realtime=False)
    for a, b in zip(fp, mx):
        scale = np.linalg.norm(a.uu)
        assert np.linalg.norm(b.uu - a.uu) / scale < 1e-5


def test_jobs_overlap_and_budget_holds():
    reqs = [S.Request(i, 256, 256, steps=60, kind="ot", mixed=True) for i in range(8)]
    budget = 4 * S.footprint_bytes(256, 256)
    res, wall = S.run_stream(reqs, budget_bytes=budget, slots=8, realtime=False)
    assert all(r.error is None for r in res), [r.error for r in res]
    # some job was admitted before another finished: the work overlapped
    spans = sorted((r.admitted, r.finished) for r in res)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    # never more than four 256^2 footprints at a time
    events = sorted([(r.admitted, 1) for r in res] + [(r.finished, -1) for r in res])
    live = peak = 0
    for _, d in events:
        live += d
        peak = max(peak, live)
    assert peak <= 4


def test_poisoned_job_fails_alone():
    # host-side fault injection: one job starts from a state with a NaN; it is
    # reported as that job's error and the others are unaffected
    jobs = _jobs(False)
    bad = S.Request(99, 128, 128, steps=20, kind="ot", keep_state=True)
    orig = bad.build

    def poisoned():
        p, uu = orig()
        uu = uu.copy()
        uu[0, 5, 7] = np.nan
        return p, uu

    bad.build = poisoned
    res, _ = S.run_stream(jobs + [bad], slots=6, realtime=False)
    byid = {r.rid: r for r in res}
    assert byid[99].error is not None and "non-finite" in byid[99].error
    alone, _ = S.run_stream(_jobs(False), slots=1, realtime=False)
    for a in alone:
        assert byid[a.rid].error is None
        np.testing.assert_array_equal(byid[a.rid].uu, a.uu)
