"""Host logic of the serving loop with a fake engine (no GPU): admission by
memory footprint and free slots, first-fit bypass, reuse of a cohort's idle
engine, LRU eviction under the budget."""
import threading
import time

import numpy as np
import pytest

from omicabelnomm_b200 import serve as S


class FakeEngine:
    live = 0
    peak = 0
    created = 0
    closed = 0
    lock = threading.Lock()

    def __init__(self, cohort, t_cap, nbytes):
        self.cohort, self.t_cap, self.nbytes = cohort.cid, t_cap, nbytes
        with FakeEngine.lock:
            FakeEngine.created += 1

    def set_traits_device(self, ptr, t):
        self.t = t

    def scan(self, ptr, mb):
        with FakeEngine.lock:
            FakeEngine.live += 1
            FakeEngine.peak = max(FakeEngine.peak, FakeEngine.live)
        time.sleep(0.002 + 1e-9 * mb * self.t)
        with FakeEngine.lock:
            FakeEngine.live -= 1
        return ("rows", self.cohort, ptr, mb, self.t)

    def device_bytes(self):
        return self.nbytes

    def close(self):
        with FakeEngine.lock:
            FakeEngine.closed += 1


def _setup(n_req=40, cohorts=5, seed=3):
    rng = np.random.Generator(np.random.PCG64(seed))
    coh = {c: S.Cohort(cid=c, rows=np.arange(100 + c), XL=np.ones((3, 100 + c), np.float32)) for c in range(cohorts)}
    reqs = []
    t_arr = 0.0
    for i in range(n_req):
        t_arr += rng.exponential(0.002)
        reqs.append(S.Request(rid=i, cohort=int(rng.integers(0, cohorts)), snp0=int(rng.integers(0, 1000)),
                              nsnp=int(rng.integers(10, 1000)), y_ptr=1000 + i, t=int(rng.integers(1, 50)),
                              arrival=t_arr))
    return coh, reqs


def _server(coh, budget, slots, nbytes=3 << 20, reuse=True):
    FakeEngine.live = FakeEngine.peak = FakeEngine.created = FakeEngine.closed = 0
    srv = S.Server(0, 200, 2000, coh, budget_bytes=budget, max_slots=slots, min_p_store=1e-3,
                   engine_factory=lambda c, t, snps=None: FakeEngine(c, t, nbytes), reuse_engines=reuse)
    srv.footprint = lambda req: 4 << 20
    return srv


@pytest.mark.parametrize("realtime", [False, True])
def test_every_request_served_within_slots_and_budget(realtime):
    coh, reqs = _setup()
    srv = _server(coh, budget=24 << 20, slots=4)
    res = srv.run(reqs, realtime=realtime)
    assert [r.rid for r in res] == list(range(len(reqs)))
    for r, q in zip(res, reqs):
        assert r.rows == ("rows", q.cohort, 4 * q.snp0 * 200, q.nsnp, q.t)   # its own cohort, range and traits
        assert r.finished >= r.admitted >= r.arrival - 1e-9
    assert FakeEngine.peak <= 4
    assert srv.peak_bytes <= 24 << 20
    summary = S.summarize(res)
    assert summary["requests"] == len(reqs) and summary["latency_p99_ms"] >= summary["latency_p50_ms"]


def test_idle_engines_are_reused_and_evicted_under_pressure():
    coh, reqs = _setup(n_req=30, cohorts=6)
    srv = _server(coh, budget=12 << 20, slots=2)
    srv.run(reqs, realtime=False)
    assert FakeEngine.created < len(reqs)          # a cohort's idle engine serves its next request
    assert srv.evictions > 0                       # 6 cohorts do not fit in the budget together
    assert srv.peak_bytes <= 12 << 20
    srv.close()


def test_request_larger_than_the_budget_is_refused():
    coh, reqs = _setup(n_req=2)
    srv = _server(coh, budget=1 << 20, slots=2)
    with pytest.raises(Exception):
        srv.run(reqs, realtime=False)


def test_footprint_grows_with_the_request():
    coh, _ = _setup()
    srv = S.Server(0, 200, 2000, coh, budget_bytes=1 << 40, max_slots=2,
                   engine_factory=lambda c, t: FakeEngine(c, t, 0))
    small = S.Request(rid=0, cohort=0, snp0=0, nsnp=100, y_ptr=0, t=2)
    big = S.Request(rid=1, cohort=0, snp0=0, nsnp=100000, y_ptr=0, t=400)
    assert srv.footprint(big) > srv.footprint(small) > 0


def test_warm_creates_the_engines_of_every_cohort():
    coh, _ = _setup(cohorts=3)
    srv = _server(coh, budget=1 << 30, slots=2)
    srv.warm("cpu", per_cohort=2)
    assert FakeEngine.created == 6
    assert sorted(s.cohort for s in srv._idle) == [0, 0, 1, 1, 2, 2]
    assert srv.max_slots == 2


def test_per_request_engines_are_created_inside_the_request_and_released():
    """Every request with its own subsample: an engine per request, created inside its
    latency (the 'engine' phase) and released when its results are out; nothing idles."""
    coh, reqs = _setup(n_req=25, cohorts=25)
    for q in reqs:
        q.cohort = q.rid
    srv = _server(coh, budget=24 << 20, slots=4, reuse=False)
    res = srv.run(reqs, realtime=True)
    assert FakeEngine.created == len(reqs) == FakeEngine.closed
    assert not srv._idle and srv.evictions == 0
    assert all("engine" in r.phases and "release" in r.phases for r in res)
    assert FakeEngine.peak <= 4


def test_requests_draw_their_own_subsample_and_covariates():
    w = S.ServeWorkload(n_total=5000, m_total=50000, requests=6, n_lo=500, n_hi=5000, seed=7)
    rng = np.random.Generator(np.random.PCG64(1))
    cohorts = [S.draw_cohort(rng, w, c) for c in range(6)]
    sizes = {c.rows.size for c in cohorts}
    assert len(sizes) > 1 and all(w.n_lo <= n <= w.n_hi for n in sizes)
    for c in cohorts:
        assert np.all(np.diff(c.rows) > 0) and c.rows.max() < w.n_total
        assert w.l_lo <= c.XL.shape[0] <= w.l_hi and c.XL.shape[1] == c.rows.size
        assert np.all(c.XL[0] == 1.0)
