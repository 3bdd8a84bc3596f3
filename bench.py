"""Benchmark: SNP x trait association tests per second on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--form mixed|plain]

Workload (one GPU, the omics-scale configuration): n = 10,000 individuals,
l = 4 covariates (intercept, sex, age, one PC), m = 500,000 SNPs (r = 1),
t = 1,000 traits with 20 missingness patterns (0-10 % missing), float32
inputs, seeded synthetic data drawn on the device.  One step = one full
association scan of that workload (5e8 tests) through the engine's C ABI
with the genotype matrix (20 GB, larger than L2) resident in HBM.

Under torchrun (N > 1) every rank scans its own equally sized workload
(SNP shards are independent, no collective on the data path: weak
scaling); the step time is the max over ranks.

The JSON line also carries:
* ``e2e``: the same scan through oa_set_traits/oa_run_snps with pinned
  HOST buffers, the host->device copies and the result download inside
  the timed region;
* ``roofline`` of the dominant kernel (the XR'Y~ GEMM with fused
  statistics) from CUDA-event times of its launches;
* ``cpu_baseline``: the reference's own CPU build (compiled from its
  sources into oracle/_ref) on a bounded sample of the same workload,
  one single-thread process per host core on disjoint SNP slices (the
  reference's MPI partition, which has no communication);
* ``clocks`` sampled with nvidia-smi during the timed region.

``--impl reference`` times only the reference CPU build (rank 0), with the
same metric and workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# the serving section runs up to 8 engines' streams at once: give the device as
# many hardware work queues as it has (must be set before CUDA starts)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

METRIC = "SNP×trait tests/s: plain FP32 vs mixed @ |Δt|≤1e-3 vs FP64; serve p50/p99"
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "omicabelnomm_ref")
WORKLOAD = dict(n=10000, l=4, r=1, m=500000, t=1000, patterns=20)


def workload_desc(m: int) -> str:
    return (f"omics-scale association scan: n={WORKLOAD['n']} individuals, l={WORKLOAD['l']} covariates, "
            f"m={m} SNPs (r=1), t={WORKLOAD['t']} traits, {WORKLOAD['patterns']} missingness patterns")


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.out = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.out,
                                     stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                c = [x.strip() for x in line.split(",")]
                if len(c) >= 9 and c[1].replace(".", "").isdigit():
                    rows.append(c)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(c[1]) for c in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for c in rows:
            for k, nm in enumerate(names):
                if c[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "samples": len(rows),
                "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# the reference's CPU build on a bounded sample
# ---------------------------------------------------------------------------
def cpu_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def prepare_reference_sample(where: str, snps_per_proc: int, procs: int):
    """Config-shaped inputs for the reference: XL, Y shared; one XR slice per process."""
    import numpy as np
    from omicabelnomm_b200 import fvformat, synth
    w = synth.scaled(1, m=snps_per_proc)
    rng = np.random.Generator(np.random.PCG64(w.seed))
    XL, xl_names = synth.covariates(rng, w)
    n, t = w.n, w.t
    obs = fvformat.obs_names(n)
    fvformat.write_fv(os.path.join(where, "XL"), XL, obs, xl_names)
    pat = rng.integers(0, w.n_patterns, t)
    frac = rng.uniform(0, w.miss_hi, w.n_patterns)
    miss = np.zeros((w.n_patterns, n), dtype=bool)
    for g in range(w.n_patterns):
        miss[g, rng.choice(n, int(round(frac[g] * n)), replace=False)] = True
    b = rng.normal(0, 1, (t, w.l))
    noise = np.sqrt(rng.uniform(w.noise_lo, w.noise_hi, t))
    Y = (b @ XL.astype(np.float64) + rng.normal(0, 1, (t, n)) * noise[:, None]).astype(np.float32)
    Y[miss[pat]] = np.nan
    fvformat.write_fv(os.path.join(where, "Y"), Y, obs, [f"ph{j + 1}" for j in range(t)])
    for q in range(procs):
        X = synth.dosages(rng, n, snps_per_proc, w.maf_lo, w.maf_hi)
        fvformat.write_fv(os.path.join(where, f"XR{q}"), X, obs, [f"snp{q}_{i}" for i in range(snps_per_proc)])
    return n, t


def time_reference(where: str, procs: int, snps_per_proc: int, t: int):
    """One step: `procs` reference processes (-t 1) on disjoint SNP slices; wall time."""
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")
    t0 = time.perf_counter()
    ps = []
    for q in range(procs):
        cmd = [REF_BIN, "-c", os.path.join(where, "XL"), "-g", os.path.join(where, f"XR{q}"), "-p",
               os.path.join(where, "Y"), "-o", os.path.join(where, f"out{q}"), "-t", "1"]
        ps.append(subprocess.Popen(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, env=env))
    rcs = [p.wait() for p in ps]
    dt = time.perf_counter() - t0
    if any(rcs):
        raise RuntimeError(f"reference exited with {rcs}")
    return procs * snps_per_proc * t / dt, dt


def reference_available():
    return os.path.exists(REF_BIN) and os.access(REF_BIN, os.X_OK)


# SNPs per reference process and step: about 5 s of single-thread work at n = 10,000, t = 1,000 (process
# start-up and input reading are then a small part of each step)
REF_SNPS_PER_PROC = 96


def cpu_baseline(snps_per_proc: int = REF_SNPS_PER_PROC, steps: int = 1):
    """The reference CPU build on a bounded sample of the workload (~10-30 s of CPU)."""
    if not reference_available():
        return None
    procs = max(1, min(cpu_cores(), 64))
    with tempfile.TemporaryDirectory(prefix="oa_ref_") as d:
        n, t = prepare_reference_sample(d, snps_per_proc, procs)
        vals = [time_reference(d, procs, snps_per_proc, t)[0] for _ in range(steps)]
    return {"value": max(vals), "unit": "tests/s", "cores": procs, "kind": "reference",
            "sample": f"{procs} processes x {snps_per_proc} SNPs x {t} traits at n={n} "
                      f"(reference CLI -t 1 per process, default thresholds, OpenBLAS 0.3.15)"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/omicabelnomm_ref was not built"}))
        return 0
    procs = max(1, min(cpu_cores(), 64))
    snps = REF_SNPS_PER_PROC
    with tempfile.TemporaryDirectory(prefix="oa_ref_") as d:
        n, t = prepare_reference_sample(d, snps, procs)
        for _ in range(args.warmup):
            time_reference(d, procs, snps, t)
        vals, times = [], []
        for _ in range(args.steps):
            v, dt = time_reference(d, procs, snps, t)
            vals.append(v)
            times.append(dt)
    tests = procs * snps * t
    value = tests * len(times) / sum(times)
    line = {"metric": METRIC, "value": value, "unit": "tests/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": workload_desc(WORKLOAD["m"]),
                                            "sample_snps": procs * snps, "partition": "one process per core"},
            "cpu_baseline": {"value": value, "unit": "tests/s", "cores": procs, "kind": "reference",
                             "sample": f"{procs} processes x {snps} SNPs x {t} traits at n={n} per step"},
            "e2e": {"value": value, "unit": "tests/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# our engine
# ---------------------------------------------------------------------------
def time_scans(eng, xr_ptr, m, steps, warmup, local, barrier, max_over_ranks):
    """Warm-up scans, then `steps` timed scans of the device-resident block."""
    import torch
    for _ in range(warmup):
        eng.run_device(xr_ptr, m)
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    launches0 = eng.launches()
    t0 = time.perf_counter()
    gemm_ms = stats_ms = block_ms = 0.0
    rows = 0
    kname = ""
    for _ in range(steps):
        r = eng.run_device(xr_ptr, m)
        ms, kname = eng.last_kernel_ms()
        gemm_ms += ms
        stats_ms += eng.last_stats_ms()
        block_ms += eng.last_block_ms()   # CUDA events on the engine's stream around the whole scan
        rows = r.count
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    barrier()
    clk = clocks.stop()
    step_s = max_over_ranks(block_ms / 1000.0 / steps)
    host_step_s = max_over_ranks(elapsed / steps)
    return dict(step_s=step_s, host_step_s=host_step_s, gemm_ms=gemm_ms / steps, stats_ms=stats_ms / steps,
                kernel=kname, launches=(eng.launches() - launches0) // steps, rows=rows, clocks=clk,
                tuning=eng.tuning())


def sgemm_peak_tflops(dev) -> float:
    """Measured FP32 (FFMA, no TF32) matrix-multiply throughput of this GPU: cuBLAS SGEMM on
    8192^3 operands, best of 5 after warm-up (the plain form's roofline denominator, as the
    cuBLAS BF16 figure is the mixed form's)."""
    import torch
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        a = torch.randn(8192, 8192, device=dev)
        b = torch.randn(8192, 8192, device=dev)
        c = a @ b
        best = float("inf")
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b, out=c)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        del a, b, c
        return 2.0 * 8192 ** 3 / best / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def max_dt(eng_a, eng_b, xr_ptr, mb):
    """max |t_a - t_b| over the tests of the first mb SNPs (both finite)."""
    import numpy as np
    out = []
    for eng in (eng_a, eng_b):
        eng.enable_dense(True)
        eng.run_device(xr_ptr, mb)
        out.append(eng.dense(mb)[2])
        eng.enable_dense(False)
    a, b = out
    ok = np.isfinite(a) & np.isfinite(b)
    return float(np.max(np.abs(a[ok] - b[ok]))) if ok.any() else None


def accuracy_vs_fp64(engines, XL, XR, Y, r, m_s):
    """Errors of each form against the FP64 oracle (the checker, oracle/oa_oracle.py) on the first
    m_s SNPs x all traits at full n, outside every timed region: max and 99.99th percentile of
    |dt|, max relative SE error, max |d beta| / SE over the tests the oracle finds regular."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oa_oracle as O
    xl = XL.cpu().numpy()
    xr = XR[:m_s * r].cpu().numpy()
    y = Y.cpu().numpy()
    l, n = xl.shape
    t = y.shape[0]
    inp = O.Inputs(XL=xl, XR=xr, Y=y, xl_names=[f"c{q}" for q in range(l)],
                   xr_names=[f"s{i}" for i in range(m_s * r)], y_names=[f"y{j}" for j in range(t)], realN=n,
                   kept=np.arange(n))
    t0 = time.perf_counter()
    D = O.solve(inp, O.Settings(r=r, storePInd=True), keep_dense=True).dense
    oracle_s = time.perf_counter() - t0
    ok = ~D.singular
    tr, ser, br = D.tstat[:, :, l:][ok], D.se[:, :, l:][ok], D.beta[:, :, l:][ok]
    out = {"sample": f"first {m_s} SNPs x {t} traits at n={n} (r={r})", "tests": int(ok.sum()),
           "max_abs_t": float(np.abs(tr).max()), "oracle_s": oracle_s}
    for name, eng in engines.items():
        eng.enable_dense(True)
        eng.run_device(XR.data_ptr(), m_s)
        b, se, tt, _ = eng.dense(m_s)
        eng.enable_dense(False)
        dt = np.abs(tt[ok] - tr)
        out[name] = {"max_dt": float(dt.max()), "p9999_dt": float(np.quantile(dt, 0.9999)),
                     "max_rel_se": float((np.abs(se[ok] - ser) / np.abs(ser)).max()),
                     "max_dbeta_over_se": float((np.abs(b[ok] - br) / np.abs(ser)).max())}
    return out


def cli_e2e(xl, xr, y, m_cli: int, precision: str):
    """The drop-in boundary end to end: the engine's CLI (omicabelnomm_b200/lib/omicabelnomm, the
    reference's flags and default thresholds) on .fvi/.fvd files of the first m_cli SNPs, written
    to RAM-backed storage and read once untimed (page cache), then one timed run: file reading,
    the scan and the _dis.txt output - the scope of the reference arm's CLI runs."""
    import numpy as np
    from omicabelnomm_b200 import engine as E
    from omicabelnomm_b200 import fvformat
    if not os.path.exists(E.CLI_PATH):
        return {"error": "CLI not built"}
    l, n = xl.shape
    t = y.shape[0]

    def need(mc):   # input files, the text output (about 80 bytes per test of 16) and headroom
        return (mc + t + l) * n * 4 * 1.3 + mc * t * 5 + (2 << 30)

    def room(path):
        return os.path.isdir(path) and shutil.disk_usage(path).free
    while m_cli > 65536 and max(room("/dev/shm") or 0, room(tempfile.gettempdir()) or 0) < need(m_cli):
        m_cli //= 2
    base = "/dev/shm" if (room("/dev/shm") or 0) > need(m_cli) else None
    if base is None and (room(tempfile.gettempdir()) or 0) < need(m_cli):
        return {"error": "no room for the input files"}
    with tempfile.TemporaryDirectory(prefix="oa_cli_", dir=base) as d:
        obs = fvformat.obs_names(n)
        fvformat.write_fv(os.path.join(d, "XL"), np.ascontiguousarray(xl), obs, [f"cov{q}" for q in range(l)])
        fvformat.write_fv(os.path.join(d, "Y"), np.ascontiguousarray(y), obs, [f"ph{j + 1}" for j in range(t)])
        fvformat.write_fv(os.path.join(d, "XR"), np.ascontiguousarray(xr[:m_cli]), obs,
                          [f"snp{i + 1}" for i in range(m_cli)])
        cmd = [E.CLI_PATH, "-c", os.path.join(d, "XL"), "-g", os.path.join(d, "XR"), "-p", os.path.join(d, "Y"),
               "-o", os.path.join(d, "out"), "--precision", precision]
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)   # page cache
        t0 = time.perf_counter()
        p = subprocess.run(cmd, check=True, capture_output=True, text=True, env=dict(os.environ, OA_TIMING="1"))
        wall = time.perf_counter() - t0
        out_bytes = os.path.getsize(os.path.join(d, "out_dis.txt"))
    sig = p.stdout.split("Number of Significant Results:")[1].split()[0] if "Significant" in p.stdout else None
    return {"value": m_cli * t / wall, "unit": "tests/s", "wall_s": wall, "precision": precision,
            "sample": f"first {m_cli} SNPs x {t} traits at n={n}: .fvd files in page cache -> _dis.txt "
                      f"({out_bytes} bytes), reference flags and default thresholds, one process",
            "significant_results": int(sig) if sig else None, "storage": base or tempfile.gettempdir(),
            "host_phases": next((ln.split("] ", 1)[1] for ln in p.stderr.splitlines() if ln.startswith("[oa timing]")),
                                None)}


def batched_section(args, dev, local, rank, barrier, max_over_ranks):
    """Batched uneven systems with interactions: n = 8,000, l = 5, r = 2
    (SNP x sex and SNP columns), t = 2,000 traits in 150 missingness-pattern
    groups of Zipf(1.2) sizes, 4,096-SNP blocks; per block one launch of each
    per-block kernel (the Schur solves of all SNP x pattern systems in one
    persistent launch), the whole scan one CUDA graph, launch parameters
    from the engine's autotuner."""
    import torch
    from omicabelnomm_b200 import engine as E
    from omicabelnomm_b200 import synth
    w = synth.scaled(3, m=args.batched_m)
    XL, XR, Y, _ = synth.generate_device(w, dev, seed_offset=rank)
    xl_host = XL.cpu().numpy()
    n, l, r, m, t = w.n, w.l, w.r, w.m, w.t
    forms = {}
    engines = {}
    for name, prec in (("mixed", E.MIXED), ("plain", E.PLAIN)):
        eng = E.Engine(n, l, r, t, m, precision=prec, device=local, min_t_store=E.t_threshold(0.1),
                       min_r2_store=1e-6)
        eng.set_tuning(chunk_snps=4096)
        eng.set_covariates(xl_host)
        eng.set_traits_device(Y.data_ptr(), t)
        t0 = time.perf_counter()
        tuned = eng.autotune(XR.data_ptr(), min(m, 32768))
        tune_s = time.perf_counter() - t0
        eng.run_device(XR.data_ptr(), m)
        R = time_scans(eng, XR.data_ptr(), m, args.steps, args.warmup, local, barrier, max_over_ranks)
        forms[name] = {"tests_per_s": m * t * int(os.environ.get("WORLD_SIZE", "1")) / R["step_s"],
                       "ms_per_step": R["step_s"] * 1e3, "gemm_ms": R["gemm_ms"], "stats_ms": R["stats_ms"],
                       "stored_rows": R["rows"], "launches_per_scan": R["launches"], "tuning": tuned,
                       "autotune_s": tune_s, "clocks": R["clocks"]}
        engines[name] = eng
    dt = max_dt(engines["mixed"], engines["plain"], XR.data_ptr(), min(m, 4096))
    acc = None
    if rank == 0 and args.accuracy_snps > 0:
        acc = accuracy_vs_fp64(engines, XL, XR, Y, r, min(m, args.accuracy_snps // 2))
    for eng in engines.values():
        eng.close()
    del XR, Y, XL
    torch.cuda.empty_cache()
    return {"workload": f"batched uneven systems: n={n}, l={l}, r={r} (SNP x sex, SNP), m={m} SNPs, t={t} traits "
                        f"in {w.n_patterns} missingness-pattern groups (Zipf({w.zipf}) sizes 1-{w.group_max}), "
                        f"4096-SNP blocks, whole scan one CUDA graph",
            "forms": forms,
            "mixed_over_plain": forms["mixed"]["tests_per_s"] / forms["plain"]["tests_per_s"],
            "max_dt_mixed_vs_plain_first_4096_snps": dt,
            "accuracy_vs_fp64": acc,
            "max_dt_vs_fp64": acc["mixed"]["max_dt"] if acc else None}


def serve_section(args, dev, local):
    """Serving loop: Poisson arrivals (20/s) of scan requests against a
    genotype matrix resident in HBM (n = 20,000 x 1,000,000 SNPs, 80 GB);
    each request draws its own subsample of n ~ U(2,000, 20,000) individuals
    with its own l ~ U{3..6} covariates, t ~ LogUniform(1, 500) traits with
    0-10 % missingness and a contiguous range of LogUniform(10k, 1M) SNPs;
    mixed form, stored rows P < 1e-3 returned to the host; admission by
    device-memory footprint, up to 8 requests on the GPU at once.  Each
    request's latency includes its engine's creation, the covariate
    factorisation, the row-subset tables, the trait block and the scan (engine
    buffers come from pools shared by all engines; a warm-up batch of other
    requests fills them, untimed).  The same requests are then offered all at
    once for the saturated throughput."""
    import torch
    from omicabelnomm_b200 import serve as S
    w = S.ServeWorkload(m_total=args.serve_m, requests=args.serve_requests)
    G = S.resident_genotypes(w, dev)
    keep = []
    reqs, cohorts = S.make_requests(w, None, dev, keep)
    ww = S.ServeWorkload(m_total=args.serve_m, requests=16, seed=w.seed + 17)
    warm_reqs, warm_cohorts = S.make_requests(ww, None, dev, keep)
    for q in warm_reqs:                      # their own ids beside the timed requests'
        q.rid += 1_000_000
        q.cohort += 1_000_000
    cohorts.update({c + 1_000_000: v for c, v in warm_cohorts.items()})
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info(dev)
    budget = int(free - (6 << 30))
    srv = S.Server(G.data_ptr(), w.n_total, w.m_total, cohorts, device=local, budget_bytes=budget, max_slots=8,
                   min_p_store=1e-3, reuse_engines=False)
    srv.run(warm_reqs, realtime=False)      # start-up, not timed: fills the buffer pools
    clocks = ClockSampler(local)
    clocks.start()
    res = srv.run(reqs, realtime=True)
    clk = clocks.stop()
    out = S.summarize(res)
    sat = S.summarize(srv.run(reqs, realtime=False))
    out.update({"workload": f"serving: resident genotypes n={w.n_total} x m={w.m_total} SNPs (float32 in HBM), "
                            f"{w.requests} requests at Poisson rate {w.rate}/s, each with its own subsample "
                            f"n_req~U({w.n_lo},{w.n_hi}) and covariates l~U{{{w.l_lo}..{w.l_hi}}}, "
                            f"t~LogU({w.t_lo:g},{w.t_hi:g}), SNP range~LogU({w.len_lo:g},{w.len_hi:g}), "
                            f"missing 0-{w.miss_hi:g}; engine creation, covariate QR and row-set build inside "
                            f"each request's latency",
                "form": "mixed", "max_concurrent": srv.max_slots, "budget_bytes": budget,
                "peak_admitted_bytes": srv.peak_bytes, "evictions": srv.evictions, "clocks": clk,
                "offered_load_tests_per_s": out["tests_per_s"],
                "saturated": {"tests_per_s": sat["tests_per_s"], "wall_s": sat["wall_s"],
                              "latency_p50_ms": sat["latency_p50_ms"], "latency_p99_ms": sat["latency_p99_ms"],
                              "note": "the same requests offered all at once"}})
    srv.close()
    del G, keep
    torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="auto", choices=["auto", "mixed", "plain"])
    ap.add_argument("--m", type=int, default=WORKLOAD["m"], help="SNPs per GPU (default: the full workload)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the engines' default tuning (profiling runs: timings under a profiler would steer "
                         "the autotuner elsewhere)")
    ap.add_argument("--batched-m", type=int, default=200000, help="SNPs of the batched workload (0: skip it)")
    ap.add_argument("--cli-snps", type=int, default=-1,
                    help="SNPs of the CLI end-to-end run (.fvd in page cache -> _dis.txt; 0: skip it; default: "
                         "the whole workload, or fewer if the files do not fit in RAM-backed or temporary storage)")
    ap.add_argument("--accuracy-snps", type=int, default=512,
                    help="SNPs of the omics-scale sample checked against the FP64 oracle outside the timed "
                         "region (half as many for the batched r = 2 workload; 0: skip)")
    ap.add_argument("--serve-requests", type=int, default=120, help="requests of the serving run (0: skip it)")
    ap.add_argument("--serve-m", type=int, default=1_000_000, help="SNPs of the resident serving matrix")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    from omicabelnomm_b200 import engine as E
    from omicabelnomm_b200 import synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    w = synth.scaled(1, m=args.m)
    XL, XR, Y, _ = synth.generate_device(w, dev, seed_offset=rank)
    n, l, m, t = w.n, w.l, w.m, w.t
    tests = m * t
    min_t = E.t_threshold(0.1)
    forms = {"mixed": E.MIXED, "plain": E.PLAIN}
    order = ["mixed", "plain"] if args.form == "auto" else [args.form]
    xl_host = XL.cpu().numpy()
    torch.cuda.synchronize()

    results = {}
    for name in order:
        try:
            eng = E.Engine(n, l, 1, t, m, precision=forms[name], device=local, min_t_store=min_t,
                           min_r2_store=1e-6)
            eng.set_covariates(xl_host)
            eng.set_traits_device(Y.data_ptr(), t)
            # launch parameters from the engine's autotuner on a sample of three default chunks (untimed)
            t0 = time.perf_counter()
            if not args.no_autotune:
                eng.autotune(XR.data_ptr(), min(m, 3 * 18944))
            tune_s = time.perf_counter() - t0
            eng.run_device(XR.data_ptr(), m)     # probe once before timing
        except E.OAError as ex:
            results[name] = {"error": str(ex)}
            continue
        results[name] = dict(engine=eng, autotune_s=tune_s,
                             **time_scans(eng, XR.data_ptr(), m, args.steps, args.warmup, local, barrier,
                                          max_over_ranks))

    valid = [k for k in order if "error" not in results[k]]
    if not valid:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "error": {k: v["error"] for k, v in results.items()}}))
        return 1
    head = valid[0]
    R = results[head]
    dt_mp = None
    if len(valid) == 2:
        dt_mp = max_dt(results["mixed"]["engine"], results["plain"]["engine"], XR.data_ptr(), min(m, 16384))
    acc = None
    if rank == 0 and args.accuracy_snps > 0:
        acc = accuracy_vs_fp64({k: results[k]["engine"] for k in valid}, XL, XR, Y, 1, min(m, args.accuracy_snps))
    for k in valid:
        if k != head:
            results[k]["engine"].close()

    # end to end through the C ABI with pinned host buffers
    xr_host = torch.empty(XR.shape, dtype=torch.float32, pin_memory=True)
    xr_host.copy_(XR)
    y_host = torch.empty(Y.shape, dtype=torch.float32, pin_memory=True)
    y_host.copy_(Y)
    del XR, Y, XL
    torch.cuda.empty_cache()
    eng = R["engine"]
    xr_np = xr_host.numpy()
    y_np = y_host.numpy()
    e2e_s = None
    d2h = 0
    link_gbs = None
    if args.e2e_steps > 0:
        # the host link's copy rate from pinned memory (the bound of the end-to-end number): best of
        # three 2 GiB copies of the genotype buffer, CUDA events
        nb = min(xr_host.numel(), (2 << 30) // 4)
        dst = torch.empty(nb, dtype=torch.float32, device=dev)
        src = xr_host.view(-1)[:nb]
        best = None
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            dst.copy_(src, non_blocking=True)
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        link_gbs = nb * 4 / (best * 1e-3) / 1e9
        del dst, src
        eng.set_traits(y_np)
        eng.run_raw(xr_np)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            eng.set_traits(y_np)
            out = eng.run_raw(xr_np)
            d2h += out.count * (16 + 12 * 1)   # stored rows come back packed by field: 16 + 12 r bytes each
        e2e_s = max_over_ranks((time.perf_counter() - t0) / args.e2e_steps)
    eng.close()
    cli = None
    if rank == 0 and world == 1 and args.cli_snps != 0:
        try:
            cli = cli_e2e(xl_host, xr_np, y_np, m if args.cli_snps < 0 else min(m, args.cli_snps), head)
        except (OSError, subprocess.CalledProcessError) as ex:
            cli = {"error": str(ex)}
    h2d = int(xr_np.nbytes + y_np.nbytes)
    del xr_host, y_host, xr_np, y_np
    torch.cuda.empty_cache()
    torch._C._host_emptyCache()   # unpin the 20 GB of host input (torch caches pinned blocks)

    batched = None
    if args.batched_m > 0:
        try:
            batched = batched_section(args, dev, local, rank, barrier, max_over_ranks)
        except E.OAError as ex:
            batched = {"error": str(ex)}

    serve = None
    if args.serve_requests > 0 and world == 1:
        try:
            serve = serve_section(args, dev, local)
        except E.OAError as ex:
            serve = {"error": str(ex)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline()
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"error": str(ex)}

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    sgemm_tf = sgemm_peak_tflops(dev)
    plain_roof = None
    if "plain" in valid:
        g = results["plain"]["gemm_ms"] / 1000.0
        ach = 2.0 * n * m * t / g / 1e12 if g > 0 else None
        plain_roof = {"bound": "fp32-simt", "kernel": results["plain"]["kernel"], "achieved": ach, "peak": sgemm_tf,
                      "unit": "TFLOP/s", "frac": (ach / sgemm_tf) if ach else None,
                      "peak_source": "measured FP32 SGEMM (cuBLAS, TF32 off, 8192^3) on this GPU in this run"}
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    flops = 2.0 * n * m * t
    gemm_s = R["gemm_ms"] / 1000.0
    achieved_tflops = flops / gemm_s / 1e12 if gemm_s > 0 else None
    if head == "mixed":
        # the GEMM runs inside back-to-back scans under the power cap: the sustained figure applies
        peak = peaks.get("bf16_tflops_sustained", 1400.0)
        peak_src = ("measured bf16 dense, sustained (seconds-long cuBLAS loop), MEASURED_PEAKS.json"
                    if "bf16_tflops_sustained" in peaks else "fallback (sustained)")
        bound = "tensor"
    else:
        peak = sgemm_tf
        peak_src = "measured FP32 SGEMM (cuBLAS, TF32 off, 8192^3) on this GPU in this run"
        bound = "fp32-simt"
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tr = json.load(f).get(R["kernel"])
            if tr:
                traffic = tr["bytes_per_launch_full"]
    except (OSError, ValueError):
        pass
    line = {
        "metric": METRIC,
        "value": tests * world / R["step_s"],
        "unit": "tests/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": R["step_s"] * 1000.0,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "bf16x3->f32" if head == "mixed" else "f32",
        "data": "synthetic",
        "config": {"workload": workload_desc(m), "form": head, "global_tests": tests * world,
                   "inputs": "genotypes resident in HBM (20 GB per GPU, larger than L2: no flush needed)",
                   "parallelism": f"independent SNP shards x{world}"},
        "e2e": ({"value": tests * world / e2e_s, "unit": "tests/s", "h2d_bytes_per_step": h2d,
                 "d2h_bytes_per_step": int(d2h / args.e2e_steps),
                 "h2d_link": {"achieved_gbs": h2d / e2e_s / 1e9, "measured_copy_gbs": link_gbs,
                              "frac": (h2d / e2e_s / 1e9) / link_gbs if link_gbs else None,
                              "note": "genotype bytes per step / step time, against a 2 GiB pinned host-to-device "
                                      "copy timed in the same run (the bound of this number)"}}
                if e2e_s else None),
        "gpu_launches": int(R["launches"] * args.steps),
        "roofline": {"bound": bound, "achieved": achieved_tflops, "peak": peak, "unit": "TFLOP/s",
                     "frac": (achieved_tflops / peak) if achieved_tflops else None, "traffic": traffic,
                     "kernel": R["kernel"], "peak_source": peak_src,
                     "algorithmic": "2*n*m*t FLOP per scan (XR'Y~), per-launch = chunk share",
                     "tensor_products": 3 if head == "mixed" else 1,
                     "frac_hardware": ((3 if head == "mixed" else 1) * achieved_tflops / peak) if achieved_tflops
                     else None},
        "cpu_baseline": cpu,
        "clocks": R["clocks"],
        "timing": "device: CUDA events on the engine's stream before the first and after the last launch "
                  "of each scan, summed over the timed scans, max over ranks",
        "forms": {k: ({"tests_per_s": tests * world / v["step_s"], "ms_per_step": v["step_s"] * 1e3,
                       "host_ms_per_step": v["host_step_s"] * 1e3, "gemm_ms": v["gemm_ms"],
                       "stats_ms": v["stats_ms"], "stored_rows": v["rows"], "tuning": v["tuning"],
                       "autotune_s": v["autotune_s"]}
                      if "error" not in v else v)
                  for k, v in results.items()},
        "plain_roofline": plain_roof,
        "e2e_cli": cli,
        "max_dt_mixed_vs_plain_first_16384_snps": dt_mp,
        "accuracy_vs_fp64": acc,
        "max_dt_vs_fp64": {"omics": acc[head]["max_dt"] if acc else None,
                           "batched_r2": (batched or {}).get("max_dt_vs_fp64")},
        "batched": batched,
        "serve": serve,
    }
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
