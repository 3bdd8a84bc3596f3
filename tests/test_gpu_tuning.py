"""Tuning parameters and the autotuner: every tuning gives the same results
(the per-SNP work does not depend on tile order, chunking or SNPs per CTA
group), and oa_autotune keeps a valid tuning."""
import numpy as np
import pytest

from omicabelnomm_b200 import engine as E
from omicabelnomm_b200 import synth

pytestmark = pytest.mark.gpu


def _data():
    w = synth.scaled(0, n=1024, m=1500, t=300, l=5, r=2, miss_mode="patterns", n_patterns=12, miss_hi=0.15,
                     seed=81)
    return w, synth.generate(w)


def _run(ds, w, prec, **tuning):
    m = ds.XR.shape[0] // w.r
    eng = E.Engine(w.n, w.l, w.r, w.t, m, precision=prec, min_t_store=E.t_threshold(0.1), min_r2_store=1e-6)
    if tuning:
        eng.set_tuning(**tuning)
    eng.set_covariates(ds.XL)
    eng.set_traits(ds.Y)
    eng.enable_dense(True)
    rows = eng.run(ds.XR)
    return eng, rows, eng.dense(m)


@pytest.mark.parametrize("prec", [E.PLAIN, E.MIXED])
def test_tunings_give_identical_results(prec):
    w, ds = _data()
    _, rows0, d0 = _run(ds, w, prec)
    variants = [dict(gemm_raster=2), dict(chunk_snps=256), dict(lean_spb=1), dict(lean_spb=4),
                dict(stats_path=1, chunk_snps=700)]
    if prec == E.MIXED:
        variants.append(dict(gemm_variant=2))
    for v in variants:
        eng, rows, d = _run(ds, w, prec, **v)
        for a, b in zip(d0, d):
            np.testing.assert_array_equal(a, b, err_msg=str(v))
        np.testing.assert_array_equal(rows0.trait, rows.trait)
        np.testing.assert_array_equal(rows0.snp, rows.snp)
        got = eng.tuning()
        for k, val in v.items():
            if k != "lean_spb":
                assert got[k] == val, (k, got)
    # the row-gather path: same numbers within FP32 summation-order differences
    _, rows_g, dg = _run(ds, w, prec, stats_path=2)
    np.testing.assert_allclose(dg[2], d0[2], rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("prec", [E.PLAIN, E.MIXED])
@pytest.mark.parametrize("spb", [1, 2])
def test_statistics_kernel_layouts_give_identical_results(prec, spb, monkeypatch):
    """One or two column buffers, with or without the row-interleaved copy of
    the set pass (the plan picks them by the weight of the set pass): same bits."""
    w, ds = _data()
    out = []
    for nbuf, xi in ((2, 1), (1, 0), (2, 0), (1, 1)):
        monkeypatch.setenv("OA_LEAN_NBUF", str(nbuf))
        monkeypatch.setenv("OA_LEAN_XI", str(xi))
        out.append(_run(ds, w, prec, lean_spb=spb, stats_path=1)[2])
    for d in out[1:]:
        for a, b in zip(out[0], d):
            np.testing.assert_array_equal(a, b)


def test_autotune_keeps_a_valid_tuning():
    import torch
    w, ds = _data()
    m = ds.XR.shape[0] // w.r
    dev = torch.device("cuda", 0)
    xr = torch.from_numpy(ds.XR).to(dev)
    y = torch.from_numpy(ds.Y).to(dev)
    eng = E.Engine(w.n, w.l, w.r, w.t, m, precision=E.MIXED, min_t_store=E.t_threshold(0.1), min_r2_store=1e-6)
    eng.set_covariates(ds.XL)
    eng.set_traits_device(y.data_ptr(), w.t)
    eng.enable_dense(True)
    eng.run_device(xr.data_ptr(), m)
    before = [a.copy() for a in eng.dense(m)]
    best = eng.autotune(xr.data_ptr(), m)
    assert best["gemm_variant"] in (1, 2, 3, 4) and best["gemm_raster"] in (1, 2) and best["stats_path"] in (1, 2)
    assert 0 < best["chunk_snps"] <= m
    eng.run_device(xr.data_ptr(), m)
    after = eng.dense(m)
    np.testing.assert_allclose(after[2], before[2], rtol=1e-4, atol=1e-4)


def test_set_tuning_rejects_out_of_range():
    eng = E.Engine(256, 3, 1, 4, 16)
    with pytest.raises(E.OAError):
        eng.set_tuning(gemm_variant=5)
    with pytest.raises(E.OAError):
        eng.set_tuning(stats_path=-1)


def test_reserve_allocates_up_front_and_changes_no_result():
    ds = synth.generate(synth.scaled(0, n=900, m=3000, t=40, seed=71))
    l, n = ds.XL.shape
    out = []
    for reserve in (True, False):
        eng = E.Engine(n, l, 1, 64, 4000, precision=E.MIXED, min_t_store=E.t_threshold(0.05), min_r2_store=1e-6)
        eng.set_covariates(ds.XL)
        if reserve:
            before = eng.device_bytes()
            eng.reserve(64, 4000)
            assert eng.device_bytes() > before
            with pytest.raises(E.OAError):
                eng.reserve(65, 10)
            with pytest.raises(E.OAError):
                eng.reserve(1, 4001)
        eng.set_traits(ds.Y)
        out.append(eng.run(ds.XR))
        eng.close()
    a, b = out
    np.testing.assert_array_equal(a.trait, b.trait)
    np.testing.assert_array_equal(a.snp, b.snp)
    np.testing.assert_array_equal(a.T, b.T)
