"""Serving on the GPU: a genotype matrix resident in device memory, scans of
cohorts (row subsets) over SNP ranges.
* the row-subset gather path of the engine matches the FP64 oracle run on
  the gathered data;
* every request gives the same stored rows and numbers alone and in a mix
  of concurrent requests (tolerance: identical, the kernels are
  deterministic)."""
import numpy as np
import pytest

import oa_oracle as O
from omicabelnomm_b200 import engine as E
from omicabelnomm_b200 import serve as S
from omicabelnomm_b200 import synth
from test_gpu_parity import T_ABS, T_REL

pytestmark = pytest.mark.gpu

N_TOTAL, M_TOTAL = 3000, 24000


@pytest.fixture(scope="module")
def resident():
    import torch
    rng = np.random.Generator(np.random.PCG64(91))
    X = synth.dosages(rng, N_TOTAL, M_TOTAL, 0.05, 0.5)            # (M, N): one SNP column per row
    X[rng.random(X.shape) < 0.001] = np.nan                      # a few missing dosages
    dev = torch.device("cuda", 0)
    return X, torch.from_numpy(X).to(dev)


def _cohorts():
    w = S.ServeWorkload(n_total=N_TOTAL, m_total=M_TOTAL, cohorts=4, n_lo=700, n_hi=N_TOTAL, seed=92)
    return w, S.make_cohorts(w)


@pytest.mark.parametrize("prec", [E.PLAIN, E.MIXED])
def test_row_subset_scan_matches_oracle(resident, prec):
    import torch
    X, Xd = resident
    _, coh = _cohorts()
    c = coh[1]
    n, l = c.rows.size, c.XL.shape[0]
    rng = np.random.Generator(np.random.PCG64(93))
    t, s0, ln = 9, 5000, 300
    Y = rng.normal(0, 1, (t, n)).astype(np.float32)
    Y[rng.random((t, n)) < 0.05] = np.nan
    eng = E.Engine(n, l, 1, t, 1000, precision=prec, store_all=True, min_t_store=E.t_threshold(0.1),
                   min_r2_store=1e-6)
    eng.set_tuning(chunk_snps=128)                                 # several chunks, each gathered
    eng.set_covariates(c.XL)
    eng.set_snp_rows(c.rows, N_TOTAL)
    y = torch.from_numpy(Y).cuda()
    eng.set_traits_device(y.data_ptr(), t)
    eng.enable_dense(True)
    eng.run_device(Xd.data_ptr() + 4 * s0 * N_TOTAL, ln)
    b, se, tt, r2 = eng.dense(ln)
    XR = np.ascontiguousarray(X[s0:s0 + ln][:, c.rows])
    inp = O.Inputs(XL=c.XL, XR=XR, Y=Y, xl_names=[f"c{i}" for i in range(l)], xr_names=[f"s{i}" for i in range(ln)],
                   y_names=[f"y{j}" for j in range(t)], realN=n, kept=np.arange(n))
    res = O.solve(inp, O.Settings(r=1, storePInd=True), keep_dense=True)
    D = res.dense
    ok = ~D.singular
    t_ref = D.tstat[:, :, l:][ok]
    dt = np.abs(tt[ok] - t_ref)
    lim = (T_REL * np.abs(t_ref) + T_ABS) if prec == E.PLAIN else np.full_like(t_ref, 1e-3)
    assert np.all(dt <= lim), f"max |dt| {dt.max():.3g}"
    # a host SNP block is refused while a row subset is set
    with pytest.raises(E.OAError):
        eng.run(XR)


def test_each_request_same_alone_and_in_the_mix(resident):
    import torch
    _, Xd = resident
    w, coh = _cohorts()
    w.requests, w.t_hi, w.len_lo, w.len_hi = 10, 80.0, 500.0, 20000.0
    keep = []
    reqs, _ = S.make_requests(w, coh, torch.device("cuda", 0), keep)
    budget = 8 << 30
    alone = {}
    srv = S.Server(Xd.data_ptr(), N_TOTAL, M_TOTAL, coh, budget_bytes=budget, max_slots=1, chunk_snps=4096,
                   min_p_store=0.05)
    for q in reqs:
        alone[q.rid] = srv.run([q], realtime=False)[0].rows
    srv.close()
    srv = S.Server(Xd.data_ptr(), N_TOTAL, M_TOTAL, coh, budget_bytes=budget, max_slots=4, chunk_snps=4096,
                   min_p_store=0.05)
    mix = srv.run(reqs, realtime=False)
    srv.close()
    assert len(mix) == len(reqs)
    assert sum(len(r.rows.trait) for r in mix) > 0
    for res in mix:
        a = alone[res.rid]
        b = res.rows
        assert len(a.trait) == len(b.trait)
        for f in ("trait", "snp", "r2", "n_used", "mask", "B", "SE", "T"):
            np.testing.assert_array_equal(getattr(a, f), getattr(b, f), err_msg=f"request {res.rid} field {f}")
    s = S.summarize(mix)
    assert s["tests"] == sum(q.t * q.nsnp for q in reqs)


def test_own_subsample_requests_same_alone_and_in_the_mix(resident):
    """The serving workload's form: every request its own subsample and covariates, its
    engine created inside the request and released after it; each request's stored rows
    are identical alone and among concurrent requests."""
    import torch
    _, Xd = resident
    w = S.ServeWorkload(n_total=N_TOTAL, m_total=M_TOTAL, requests=8, n_lo=700, n_hi=N_TOTAL, t_hi=60.0,
                        len_lo=500.0, len_hi=20000.0, seed=96)
    keep = []
    reqs, coh = S.make_requests(w, None, torch.device("cuda", 0), keep)
    assert len(coh) == len(reqs) and len({c.rows.size for c in coh.values()}) > 1
    kw = dict(budget_bytes=8 << 30, chunk_snps=4096, min_p_store=0.05, reuse_engines=False)
    srv = S.Server(Xd.data_ptr(), N_TOTAL, M_TOTAL, coh, max_slots=1, **kw)
    alone = {q.rid: srv.run([q], realtime=False)[0].rows for q in reqs}
    srv.close()
    srv = S.Server(Xd.data_ptr(), N_TOTAL, M_TOTAL, coh, max_slots=4, **kw)
    mix = srv.run(reqs, realtime=False)
    assert not srv._idle
    srv.close()
    for res in mix:
        a, b = alone[res.rid], res.rows
        for f in ("trait", "snp", "r2", "n_used", "mask", "B", "SE", "T"):
            np.testing.assert_array_equal(getattr(a, f), getattr(b, f), err_msg=f"request {res.rid} field {f}")
        assert res.phases["engine"] > 0


@pytest.mark.parametrize("prec", [E.PLAIN, E.MIXED])
def test_row_subset_gives_the_numbers_of_the_gathered_block(resident, prec):
    """A scan over a row subset of the resident matrix (gathered by the
    column-statistics kernel in the mixed form, by a gather kernel in the
    FP32 form) returns bit-identical statistics to a scan of the gathered
    block as a contiguous device array."""
    import torch
    X, Xd = resident
    _, coh = _cohorts()
    c = coh[2]
    n, l = c.rows.size, c.XL.shape[0]
    rng = np.random.Generator(np.random.PCG64(94))
    t, s0, ln = 21, 7001, 777
    Y = rng.normal(0, 1, (t, n)).astype(np.float32)
    Y[rng.random((t, n)) < 0.05] = np.nan
    y = torch.from_numpy(Y).cuda()
    out = []
    for subset in (True, False):
        eng = E.Engine(n, l, 1, t, 1000, precision=prec, store_all=True, min_t_store=E.t_threshold(0.1),
                       min_r2_store=1e-6)
        eng.set_tuning(chunk_snps=256)
        eng.set_covariates(c.XL)
        eng.set_traits_device(y.data_ptr(), t)
        eng.enable_dense(True)
        if subset:
            eng.set_snp_rows(c.rows, N_TOTAL)
            eng.run_device(Xd.data_ptr() + 4 * s0 * N_TOTAL, ln)
        else:
            blk = torch.from_numpy(np.ascontiguousarray(X[s0:s0 + ln][:, c.rows])).cuda()
            eng.run_device(blk.data_ptr(), ln)
        out.append(eng.dense(ln))
        eng.close()
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("prec", [E.PLAIN, E.MIXED])
def test_single_buffered_unaligned_columns_match_oracle(prec):
    """n = 26,003: one column buffer per CTA (two do not fit in shared memory)
    and columns that are not 16-byte aligned (element-wise staging)."""
    ds = synth.generate(synth.scaled(0, n=26003, m=40, t=3, seed=95))
    l, n = ds.XL.shape
    eng = E.Engine(n, l, 1, 3, 40, precision=prec, store_all=True, min_t_store=E.t_threshold(0.1),
                   min_r2_store=1e-6)
    eng.set_covariates(ds.XL)
    eng.set_traits(ds.Y)
    eng.enable_dense(True)
    eng.run(ds.XR)
    b, se, tt, r2 = eng.dense(40)
    inp = O.Inputs(XL=ds.XL, XR=ds.XR, Y=ds.Y, xl_names=ds.xl_names, xr_names=ds.xr_names, y_names=ds.y_names,
                   realN=n, kept=np.arange(n))
    res = O.solve(inp, O.Settings(r=1, storePInd=True), keep_dense=True)
    D = res.dense
    ok = ~D.singular
    t_ref = D.tstat[:, :, l:][ok]
    dt = np.abs(tt[ok] - t_ref)
    lim = (T_REL * np.abs(t_ref) + T_ABS) if prec == E.PLAIN else np.full_like(t_ref, 1e-3)
    assert np.all(dt <= lim), f"max |dt| {dt.max():.3g}"
