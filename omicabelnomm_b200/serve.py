"""Serving loop: association scans against a genotype matrix kept resident in
HBM, with continuous batching.

A request names a cohort (a subset of the resident individuals with its own
covariates: in the serving workload every request draws its own), brings its
traits (device memory, NaN = missing) and a contiguous SNP range.  The loop

* admits waiting requests in arrival order whenever a slot is free and the
  request's device-memory footprint fits the budget (first fit: a large
  request at the head does not block smaller ones behind it, for at most
  max_bypass_s seconds);
* runs every admitted request on its own host thread and its own engine
  (own CUDA streams), so the kernels of concurrent requests overlap on the
  device; the ctypes calls release the GIL;
* creates the request's engine inside its latency (covariate factorisation,
  row subset, reservations) unless an idle engine of the same cohort holds
  its traits (reuse_engines: requests that repeat a cohort); engine buffers
  come from pools shared by all engines (device memory from the device's
  stream-ordered pool, page-locked host buffers from the engine library's
  pool), so a new engine allocates little; idle engines are evicted, least
  recently used first, when an admission needs their memory;
* reports per-request latency (arrival to results on the host), queueing
  and run time, and the aggregate tests/s.

There is no counterpart in the reference, which runs one scan per process
(src/main.cpp:440-500).  Each request's numbers are the engine's own: a
request gives the same result alone and in a mix.
"""
from __future__ import annotations

import os
import threading
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import engine as E

# Concurrent requests run on separate streams; with the default 8 hardware
# work queues, streams share queues and one request's queued chunks hold up
# another's kernels.  Effective only when set before the process starts CUDA.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")


@dataclass
class Cohort:
    cid: int
    rows: np.ndarray          # ascending indices of the cohort's individuals in the resident matrix
    XL: np.ndarray            # (l, n) covariates of those individuals


@dataclass
class Request:
    rid: int
    cohort: int
    snp0: int                 # first SNP of the range
    nsnp: int                 # SNPs in the range
    y_ptr: int                # device pointer of the traits, (t, n) float32 row-major (column-major n x t)
    t: int
    arrival: float = 0.0      # seconds after the start of the run


@dataclass
class Result:
    rid: int
    rows: E.StoredRows
    tests: int
    arrival: float
    admitted: float
    finished: float
    phases: dict = field(default_factory=dict)   # seconds: engine (creation), traits, scan (incl. results to host)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def queued(self) -> float:
        return self.admitted - self.arrival


@dataclass
class _Slot:
    engine: E.Engine
    cohort: int
    l: int
    t_cap: int
    bytes: int = 0


class Server:
    """Continuous-batching scan server over a resident genotype matrix.

    geno_ptr: device pointer of the genotypes, column-major n_total x m_total
    (float32, r = 1: one column per SNP, NaN = missing dosage).
    """

    def __init__(self, geno_ptr: int, n_total: int, m_total: int, cohorts: Dict[int, Cohort], *,
                 device: int = 0, budget_bytes: int, max_slots: int = 8, precision: int = E.MIXED,
                 chunk_snps: int = 0, min_p_store: float = 1e-3, max_snps: Optional[int] = None,
                 engine_factory=None, t_cap_min: int = 64, reuse_engines: bool = True):
        self.geno_ptr = geno_ptr
        self.n_total = n_total
        self.m_total = m_total
        self.cohorts = cohorts
        self.device = device
        self.budget = budget_bytes
        self.max_slots = max_slots
        self.precision = precision
        self.chunk = chunk_snps
        self.min_p_store = min_p_store
        self.max_snps = max_snps or m_total
        self.engine_factory = engine_factory or self._engine
        self.peak_bytes = 0             # largest admitted + idle footprint seen
        self.evictions = 0
        self.max_bypass_s = 2.0         # later requests may pass a waiting one for this long
        self.t_cap_min = t_cap_min      # trait capacity of a new engine (larger ones are reused more)
        self.reuse_engines = reuse_engines   # keep an engine for later requests of its cohort
        self._anchor = None
        if engine_factory is None:
            # a small engine held for the server's lifetime: the device keeps the freed memory of
            # per-request engines in its pool (the engine library returns the pool's memory when the
            # last engine on a device goes)
            self._anchor = E.Engine(64, 1, 1, 1, 1, precision=precision, device=device)
        self._lock = threading.Condition()
        self._idle: List[_Slot] = []    # idle engines, least recently used first (several per cohort allowed)
        self._active_bytes = 0
        self._active = 0

    # largest SNP chunk an engine picks by itself (whole waves of 128-SNP tiles, about 16,384 SNPs)
    AUTO_CHUNK_BOUND = 32768

    # -- memory ---------------------------------------------------------------
    def footprint(self, req: Request) -> int:
        """Upper estimate of the device bytes an engine needs for this request."""
        c = self.cohorts[req.cohort]
        n = c.rows.size
        l = c.XL.shape[0]
        n_pad = (n + 63) // 64 * 64
        t = req.t
        chunk = min(self.chunk if self.chunk > 0 else self.AUTO_CHUNK_BOUND, req.nsnp)
        traits = t * n * 4 + t * n_pad * 8 + t * (64 + 8 * l)
        sets = l * (1 + 2 * t) * n_pad * 8 + n * 8 * 2           # B2 (+BF16) for the worst case of set counts
        chunks = chunk * n * 4 + chunk * n_pad * 4 + chunk * (l * (1 + 2 * t) + 2 * t + 16) * 8
        tests = t * req.nsnp
        p_store = float(self.min_p_store)
        cap = max(1 << 16, int(tests * min(1.0, 1.2 * p_store + 1e-3)))
        rows = 2 * cap * 80 + cap * 24 + (64 << 20)
        return int(traits + sets + chunks + rows + (32 << 20))

    def _idle_bytes(self) -> int:
        return sum(s.bytes for s in self._idle)

    # -- engines --------------------------------------------------------------
    def _take_engine(self, req: Request) -> Optional[_Slot]:
        """The most recently used idle engine of the request's cohort that holds its traits (caller holds the lock)."""
        if not self.reuse_engines:
            return None
        for q in range(len(self._idle) - 1, -1, -1):
            slot = self._idle[q]
            if slot.cohort == req.cohort and slot.t_cap >= req.t:
                return self._idle.pop(q)
        return None

    def _engine(self, cohort: Cohort, t_cap: int, snps: Optional[int] = None):
        """The default engine factory: an engine over the cohort's rows of the resident matrix,
        for trait blocks of up to t_cap traits and SNP ranges of up to `snps` SNPs."""
        n, l = cohort.rows.size, cohort.XL.shape[0]
        snps = snps or self.max_snps
        eng = E.Engine(n, l, 1, t_cap, snps, precision=self.precision, device=self.device,
                       min_t_store=E.t_threshold(self.min_p_store), min_r2_store=1e-6)
        if self.chunk > 0:
            eng.set_tuning(chunk_snps=self.chunk)
        eng.set_covariates(cohort.XL)
        eng.set_snp_rows(cohort.rows, self.n_total)
        eng.reserve(t_cap, snps)              # no allocations once it scans
        return eng

    def _new_engine(self, req: Request) -> _Slot:
        c = self.cohorts[req.cohort]
        if self.reuse_engines:               # kept for later requests: room for any of them
            t_cap = max(req.t, self.t_cap_min)
            eng = self.engine_factory(c, t_cap)
        else:                                # this request only: its own sizes
            t_cap = req.t
            eng = self.engine_factory(c, t_cap, req.nsnp)
        return _Slot(engine=eng, cohort=req.cohort, l=c.XL.shape[0], t_cap=t_cap)

    # -- one request ----------------------------------------------------------
    def _serve_one(self, req: Request, need: int, slot: Optional[_Slot], t_start: float, arrival: float,
                   admitted: float, results: List[Result], errors: List[BaseException]):
        try:
            ph = {}
            t0 = time.perf_counter()
            if slot is None:
                slot = self._new_engine(req)
            t1 = time.perf_counter()
            eng = slot.engine
            eng.set_traits_device(req.y_ptr, req.t)
            t2 = time.perf_counter()
            ptr = self.geno_ptr + 4 * req.snp0 * self.n_total
            out = eng.scan(ptr, req.nsnp)
            t3 = time.perf_counter()
            ph = {"engine": t1 - t0, "traits": t2 - t1, "scan": t3 - t2}
            finished = t3 - t_start
            slot.bytes = eng.device_bytes()
            if not self.reuse_engines:      # its buffers go back to the pools (after the results are out)
                slot.engine.close()
                slot = None
                ph["release"] = time.perf_counter() - t3
            results.append(Result(rid=req.rid, rows=out, tests=req.t * req.nsnp, arrival=arrival,
                                  admitted=admitted, finished=finished, phases=ph))
        except BaseException as ex:  # reported to the caller of run()
            errors.append(ex)
            if slot is not None:
                slot.engine.close()
                slot = None
        with self._lock:
            self._active -= 1
            self._active_bytes -= need
            if slot is not None:
                self._idle.append(slot)
            self._lock.notify_all()

    # -- the loop -------------------------------------------------------------
    def run(self, requests: List[Request], realtime: bool = True) -> List[Result]:
        """Serve `requests`.  With realtime, each request arrives at its
        `arrival` time (latency counts from then); otherwise all arrive at
        once at the start."""
        reqs = sorted(requests, key=lambda q: q.arrival)
        results: List[Result] = []
        errors: List[BaseException] = []
        threads: List[threading.Thread] = []
        waiting: List[Request] = []
        t_start = time.perf_counter()
        nxt = 0
        with self._lock:
            while nxt < len(reqs) or waiting or self._active:
                now = time.perf_counter() - t_start
                while nxt < len(reqs) and (not realtime or reqs[nxt].arrival <= now):
                    waiting.append(reqs[nxt])
                    nxt += 1
                admitted_any = False
                for req in list(waiting):
                    if self._active >= self.max_slots:
                        break
                    if req is not waiting[0] and (waiting[0].arrival if realtime else 0.0) + self.max_bypass_s < now:
                        break                                   # the head has waited long enough: no more bypassing
                    need = self.footprint(req)
                    slot = self._take_engine(req)
                    if slot is not None:
                        need = max(need, slot.bytes)            # the engine's memory moves from idle to active
                    # evict idle engines (least recently used first) until the request fits
                    while self._active_bytes + self._idle_bytes() + need > self.budget and self._idle:
                        victim = self._idle.pop(0)
                        victim.engine.close()
                        self.evictions += 1
                    if self._active_bytes + self._idle_bytes() + need > self.budget:
                        if slot is not None:
                            self._idle.append(slot)
                        if self._active == 0 and not self._idle:
                            raise E.OAError(6, f"request {req.rid} needs {need} bytes, budget {self.budget}")
                        continue
                    waiting.remove(req)
                    self._active += 1
                    self._active_bytes += need
                    self.peak_bytes = max(self.peak_bytes, self._active_bytes + self._idle_bytes())
                    admitted = time.perf_counter() - t_start
                    arrival = req.arrival if realtime else 0.0
                    th = threading.Thread(target=self._serve_one,
                                          args=(req, need, slot, t_start, arrival, admitted, results, errors),
                                          daemon=True)
                    threads.append(th)
                    th.start()
                    admitted_any = True
                if errors:
                    break
                if not admitted_any:
                    timeout = None
                    if nxt < len(reqs) and realtime:
                        timeout = max(0.0, reqs[nxt].arrival - (time.perf_counter() - t_start))
                    if self._active or timeout is not None:
                        self._lock.wait(timeout=timeout if timeout is not None else 0.5)
        for th in threads:
            th.join()
        if errors:
            raise errors[0]
        return sorted(results, key=lambda r: r.rid)

    def warm(self, device=None, per_cohort: int = 1):
        """Create and keep `per_cohort` engines for every cohort (covariate
        factorisation, buffers) by serving 1-trait, 1000-SNP requests, the
        engines of a cohort at the same time (so that each gets its own)."""
        import torch
        keep, reqs = [], []
        for k in range(per_cohort):
            for cid, c in self.cohorts.items():
                y = torch.randn((1, c.rows.size), device=device if device is not None else f"cuda:{self.device}")
                keep.append(y)
                reqs.append(Request(rid=-1 - len(reqs), cohort=cid, snp0=0, nsnp=min(1000, self.m_total),
                                    y_ptr=y.data_ptr(), t=1))
        saved, self.max_slots = self.max_slots, max(self.max_slots, len(reqs))
        try:
            self.run(sorted(reqs, key=lambda q: q.cohort), realtime=False)
        finally:
            self.max_slots = saved
        if torch.cuda.is_available():
            torch.cuda.synchronize()

    def close(self):
        with self._lock:
            for s in self._idle:
                s.engine.close()
            self._idle.clear()
            if self._anchor is not None:
                self._anchor.close()
                self._anchor = None


def summarize(results: List[Result]) -> dict:
    """p50/p99 latency, queueing, aggregate tests/s of a run."""
    lat = np.array([r.latency for r in results])
    q = np.array([r.queued for r in results])
    tests = sum(r.tests for r in results)
    t0 = min(r.arrival for r in results)
    t1 = max(r.finished for r in results)
    phases = {}
    for k in ("engine", "traits", "scan", "release"):
        v = np.array([r.phases.get(k, 0.0) for r in results])
        phases[k + "_p50_ms"] = float(np.percentile(v, 50) * 1e3)
        phases[k + "_p99_ms"] = float(np.percentile(v, 99) * 1e3)
    return {"requests": len(results), "tests": int(tests), "wall_s": t1 - t0, "phases": phases,
            "tests_per_s": tests / (t1 - t0) if t1 > t0 else None,
            "latency_p50_ms": float(np.percentile(lat, 50) * 1e3),
            "latency_p99_ms": float(np.percentile(lat, 99) * 1e3),
            "latency_max_ms": float(lat.max() * 1e3),
            "queue_p50_ms": float(np.percentile(q, 50) * 1e3),
            "queue_p99_ms": float(np.percentile(q, 99) * 1e3)}


# ---------------------------------------------------------------------------
# synthetic request stream (the serving workload)
# ---------------------------------------------------------------------------
@dataclass
class ServeWorkload:
    n_total: int = 20000
    m_total: int = 1_000_000
    rate: float = 20.0          # Poisson arrivals per second
    requests: int = 120
    cohorts: int = 0            # 0: every request draws its own subsample and covariates
    n_lo: int = 2000
    n_hi: int = 20000
    t_lo: float = 1.0
    t_hi: float = 500.0
    len_lo: float = 1e4
    len_hi: float = 1e6
    l_lo: int = 3
    l_hi: int = 6
    miss_hi: float = 0.10
    seed: int = 4004


def draw_cohort(rng, w: ServeWorkload, cid: int) -> Cohort:
    """n ~ U(n_lo, n_hi) individuals of the resident matrix, l ~ U{l_lo..l_hi} covariates
    (intercept, sex, age, PCs)."""
    n = int(rng.integers(w.n_lo, w.n_hi + 1))
    rows = np.sort(rng.choice(w.n_total, n, replace=False)).astype(np.int32)
    l = int(rng.integers(w.l_lo, w.l_hi + 1))
    cols = [np.ones(n), (rng.random(n) < 0.5).astype(np.float64), rng.normal(50, 10, n)]
    for _ in range(l - 3):
        cols.append(rng.normal(0, 1, n))
    return Cohort(cid=cid, rows=rows, XL=np.stack(cols[:l]).astype(np.float32))


def make_cohorts(w: ServeWorkload) -> Dict[int, Cohort]:
    """w.cohorts fixed cohorts that requests share (make_requests with cohorts)."""
    rng = np.random.Generator(np.random.PCG64(w.seed))
    return {c: draw_cohort(rng, w, c) for c in range(w.cohorts)}


def make_requests(w: ServeWorkload, cohorts: Optional[Dict[int, Cohort]], device, keep: list):
    """(requests, cohorts): requests with Poisson arrivals; traits drawn on the device (kept
    alive in `keep`): t ~ LogUniform(t_lo, t_hi) traits Y = XL b + N(0, 1) with b ~ N(0, 1)
    over the cohort's covariates, SNP range length ~ LogUniform(len_lo, len_hi), 1-4
    missingness patterns per request with 0-miss_hi missing each.  With cohorts None every
    request draws its own subsample and covariates (draw_cohort; cohort id = request id);
    otherwise requests pick one of the given cohorts."""
    import torch
    rng = np.random.Generator(np.random.PCG64(w.seed + 1))
    g = torch.Generator(device=device)
    g.manual_seed(w.seed)
    arrivals = np.cumsum(rng.exponential(1.0 / w.rate, w.requests))
    arrivals -= arrivals[0]
    reqs = []
    own = cohorts is None
    if own:
        cohorts = {}
    for i in range(w.requests):
        if own:
            cid = i
            cohorts[cid] = draw_cohort(rng, w, cid)
        else:
            cid = int(rng.integers(0, len(cohorts)))
        n = cohorts[cid].rows.size
        t = max(1, int(round(np.exp(rng.uniform(np.log(w.t_lo), np.log(w.t_hi))))))
        ln = int(round(np.exp(rng.uniform(np.log(w.len_lo), np.log(min(w.len_hi, w.m_total))))))
        ln = max(1, min(ln, w.m_total))
        s0 = int(rng.integers(0, w.m_total - ln + 1))
        XL = torch.from_numpy(cohorts[cid].XL).to(device)
        b = torch.randn((t, XL.shape[0]), generator=g, device=device)
        Y = b @ XL + torch.randn((t, n), generator=g, device=device)
        G = int(rng.integers(1, 5))
        pat = torch.as_tensor(rng.integers(0, G, t), device=device)
        frac = torch.as_tensor(rng.uniform(0, w.miss_hi, G), device=device, dtype=torch.float32)
        miss = torch.rand((G, n), generator=g, device=device) < frac[:, None]
        Y = torch.where(miss[pat], torch.full_like(Y, float("nan")), Y).contiguous()
        keep.append(Y)
        reqs.append(Request(rid=i, cohort=cid, snp0=s0, nsnp=ln, y_ptr=Y.data_ptr(), t=t,
                            arrival=float(arrivals[i])))
    return reqs, cohorts


def resident_genotypes(w: ServeWorkload, device, snp_chunk: int = 16384):
    """The resident matrix on the device: m_total SNP columns of n_total dosages
    (Binomial(2, maf) + U(-0.05, 0.05), clipped to [0, 2], rounded to 0.001,
    maf ~ U(0.05, 0.5)), float32, drawn with torch in chunks."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(w.seed * 7919 + 1)
    X = torch.empty((w.m_total, w.n_total), dtype=torch.float32, device=device)
    maf = 0.05 + 0.45 * torch.rand(w.m_total, generator=g, device=device)
    for c0 in range(0, w.m_total, snp_chunk):
        c1 = min(w.m_total, c0 + snp_chunk)
        p = maf[c0:c1, None]
        x = (torch.rand((c1 - c0, w.n_total), generator=g, device=device) < p).to(torch.float32)
        x += (torch.rand((c1 - c0, w.n_total), generator=g, device=device) < p).to(torch.float32)
        x += 0.1 * torch.rand((c1 - c0, w.n_total), generator=g, device=device) - 0.05
        X[c0:c1] = torch.round(x.clamp_(0.0, 2.0) * 1000.0) / 1000.0
        del x
    return X
