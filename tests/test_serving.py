"""Host logic of the serving layer (no GPU): admission by HBM footprint,
first-come-first-served order, concurrency bounded by the slots, request
streams and the latency summary."""
import threading
import time

import numpy as np

from mhd2dcfdfftw_open_b200 import serving as S


class FakeServer(S.Server):
    """Jobs sleep instead of running on a GPU; records what ran together."""

    def __init__(self, *a, **k):
        self.lock = threading.Lock()
        self.active = []
        self.peak_bytes = 0.0
        self.peak_jobs = 0
        self.order = []
        super().__init__(*a, **k)

    def _run(self, req, admitted):
        fp = S.footprint_bytes(req.nx, req.ny)
        with self.lock:
            self.active.append(fp)
            self.order.append(req.rid)
            self.peak_bytes = max(self.peak_bytes, sum(self.active))
            self.peak_jobs = max(self.peak_jobs, len(self.active))
        time.sleep(0.002 * req.steps / 100)
        with self.lock:
            self.active.remove(fp)
        return S.Result(req.rid, req.nx * req.ny, req.steps, req.arrival, admitted,
                        self.clock(), 1e-3, 1.0)


def test_footprint_counts_the_reference_arrays():
    assert S.footprint_bytes(256, 256) == 64 * 256 * 256 * 8 + (8 << 20)
    assert S.footprint_bytes(256, 256, nvar=9) == 69 * 256 * 256 * 8 + (8 << 20)


def test_admission_respects_budget_and_slots():
    reqs = S.draw_requests(40, seed=7, rate=0.0, sizes=S.ENSEMBLE_SIZES,
                           inverse_cells=False, steps=(100, 300))
    budget = 3 * S.footprint_bytes(1024, 1024)
    srv = FakeServer(budget, slots=5)
    srv.start_clock()
    for r in reqs:
        srv.submit(r)
    srv.drain()
    assert len(srv.results) == 40
    assert srv.peak_bytes <= budget
    assert 1 < srv.peak_jobs <= 5
    assert srv.order == sorted(srv.order)  # first come, first served


def test_oversized_request_is_rejected():
    srv = FakeServer(S.footprint_bytes(256, 256), slots=1)
    try:
        r = S.Request(0, 512, 512, 10)
        try:
            srv.submit(r)
            raise AssertionError("accepted a job above the budget")
        except ValueError:
            pass
    finally:
        srv.drain()


def test_request_stream_is_seeded_and_poisson():
    a = S.draw_requests(500, seed=5, rate=20.0)
    b = S.draw_requests(500, seed=5, rate=20.0)
    assert [(r.nx, r.steps, r.kind, r.arrival) for r in a] == \
           [(r.nx, r.steps, r.kind, r.arrival) for r in b]
    gaps = np.diff([0.0] + [r.arrival for r in a])
    assert abs(gaps.mean() - 1 / 20.0) < 0.01
    cells = np.array([r.nx * r.ny for r in a])
    # probability proportional to 1/cells: the smallest size dominates
    assert (cells == 128 * 128).mean() > 0.5
    assert all(100 <= r.steps <= 2000 for r in a)
    assert all(0.0 <= r.di <= 0.1 and 1e-4 <= r.eta <= 1e-3 and r.eta == r.nu for r in a)


def test_summary_percentiles():
    res = [S.Result(i, 100, 10, 0.0, 0.0, float(i + 1), 1e-3, 1.0) for i in range(100)]
    s = S.summarize(res, 100.0)
    assert s["p50_latency_s"] == np.percentile(np.arange(1, 101), 50)
    assert s["p99_latency_s"] == np.percentile(np.arange(1, 101), 99)
    assert s["cell_updates_per_s"] == 100 * 100 * 10 / 100.0


def test_router_places_whole_jobs_across_devices():
    reqs = S.draw_requests(60, seed=9, rate=0.0, sizes=S.ENSEMBLE_SIZES,
                           inverse_cells=False, steps=(100, 200))
    budget = 2 * S.footprint_bytes(1024, 1024)
    r = S.Router([0, 1], budget, slots=3, server_cls=FakeServer)
    r.start_clock()
    for q in reqs:
        r.submit(q)
    res = r.drain()
    assert sorted(x.rid for x in res) == list(range(60))   # every job ran exactly once
    assert set(r.placement.values()) == {0, 1}            # both devices used
    for srv in r.servers:
        assert srv.peak_bytes <= budget                    # each device keeps its budget
    work = [sum(S.footprint_bytes(q.nx, q.ny) for q in reqs if r.placement[q.rid] == d)
            for d in (0, 1)]
    assert max(work) < 2.0 * min(work)                     # roughly balanced by bytes


def test_run_stream_over_a_router(monkeypatch):
    monkeypatch.setattr(S, "Server", FakeServer)
    reqs = S.draw_requests(12, seed=2, rate=0.0, sizes=((128, 128), (256, 256)),
                           inverse_cells=False, steps=(100, 100))
    res, wall = S.run_stream(reqs, budget_bytes=1e12, slots=2, realtime=False, devices=[0, 1])
    assert [r.rid for r in res] == list(range(12)) and wall > 0


def test_queued_request_can_be_cancelled():
    srv = FakeServer(S.footprint_bytes(256, 256), slots=1)
    srv.start_clock()
    reqs = [S.Request(i, 256, 256, steps=2000) for i in range(4)]   # the first runs ~40 ms
    for r in reqs:
        srv.submit(r)
    assert srv.cancel(3) is True          # still queued behind the budget
    assert srv.cancel(99) is False        # unknown
    srv.drain()
    assert sorted(r.rid for r in srv.results) == [0, 1, 2]


def test_job_record_fields():
    r = S.Result(3, 128 * 128, 100, 1.0, 2.0, 4.0, 1e-3, 0.5, None, None, 0.1)
    rec = r.record()
    assert rec["latency_s"] == 3.0 and rec["queued_s"] == 1.0
    assert rec["cell_updates_per_s"] == 128 * 128 * 100 / 2.0
    assert rec["cross_helicity"] == 0.1 and rec["error"] is None


class _BrokenRequest(S.Request):
    def build(self):
        raise RuntimeError("initial condition could not be built")


def test_failed_build_is_the_jobs_error_and_releases_its_bytes():
    # the real Server._run: the build raises before any device work
    budget = S.footprint_bytes(256, 256)
    srv = S.Server(budget, slots=1)
    srv.start_clock()
    srv.submit(_BrokenRequest(0, 256, 256, 10))
    srv.submit(_BrokenRequest(1, 256, 256, 10))   # fits only once the first has released
    srv.drain()                                   # returns: nothing leaked
    assert sorted(r.rid for r in srv.results) == [0, 1]
    assert all("could not be built" in r.error for r in srv.results)
    assert srv._reserved == 0


def test_summary_counts_finite_jobs_apart():
    res = [S.Result(i, 100, 10, 0.0, 0.0, float(i + 1), 1e-3, 1.0,
                    None, "non-finite state (NaN or Inf) at the end of the job" if i % 4 == 0 else None)
           for i in range(100)]
    s = S.summarize(res, 100.0)
    assert s["nonfinite"] == 25 and s["finite_jobs"] == 75
    assert s["cell_updates_per_s"] == 100 * 100 * 10 / 100.0
    assert s["finite_cell_updates_per_s"] == 75 * 100 * 10 / 100.0
    ok_lat = [float(i + 1) for i in range(100) if i % 4]
    assert s["finite_p50_latency_s"] == np.percentile(ok_lat, 50)


def test_router_ranks_devices_on_current_load():
    # device 0 has finished its earlier work: a new request goes there again
    budget = 4 * S.footprint_bytes(512, 512)
    r = S.Router([0, 1], budget, slots=1, server_cls=FakeServer)
    r.start_clock()
    r.submit(S.Request(0, 512, 512, 100))
    r.servers[0].drain()                      # device 0 idle again, device 1 never used
    r.servers[0] = FakeServer(budget, slots=1, device=0)
    r.servers[0].start_clock()
    r.submit(S.Request(1, 256, 256, 2000))    # ties: lower device
    r.submit(S.Request(2, 256, 256, 2000))    # device 0 now busy: goes to 1
    assert r.placement == {0: 0, 1: 0, 2: 1}
    r.drain()
