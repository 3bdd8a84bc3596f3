"""GPU parity of the mixed-precision form (tcgen05 BF16 hi/lo, 3 products,
FP32 accumulate) against the FP64 oracle.  Target: max |dt| <= 1e-3."""
import numpy as np
import pytest

import oa_oracle as O
from omicabelnomm_b200 import engine as E
from omicabelnomm_b200 import synth
from test_gpu_parity import CASES, engine_run, oracle_dense

pytestmark = pytest.mark.gpu

T_ABS_MIXED = 1e-3          # |t_mixed - t_fp64| <= 1e-3 (plus 1e-4 relative for very large t)
T_REL_MIXED = 1e-4


@pytest.mark.parametrize("case", ["r1_uniform", "r1_patterns", "r1_xrnan", "r1_collinear", "r2_complete",
                                  "r2_missing"])
def test_mixed_dense_matches_fp64_oracle(case):
    w = synth.scaled(0, **CASES[case])
    ds = synth.generate(w)
    res, inp, s = oracle_dense(ds, w.r)
    eng, rows, (b, se, tt, r2) = engine_run(ds, w.r, precision=E.MIXED)
    D = res.dense
    ok = ~D.singular
    t_ref = D.tstat[:, :, res.l:][ok]
    dt = np.abs(tt[ok] - t_ref)
    lim = T_ABS_MIXED + T_REL_MIXED * np.abs(t_ref)
    assert np.all(dt <= lim), f"max |dt| {dt.max():.3g}"
    assert np.allclose(se[ok], D.se[:, :, res.l:][ok], rtol=1e-4, atol=0)


def test_mixed_matches_plain_on_stored_rows():
    ds = synth.generate(synth.scaled(0, n=1000, m=700, t=300, l=4, miss_mode="patterns", n_patterns=7, seed=51))
    _, rp, (bp, sp, tp, r2p) = engine_run(ds, 1, precision=E.PLAIN)
    _, rm, (bm, sm, tm, r2m) = engine_run(ds, 1, precision=E.MIXED)
    assert np.nanmax(np.abs(tp - tm)) < 1e-3
    assert rp.tests == rm.tests


def test_mixed_multiple_tiles_and_ragged_edges():
    """t and m not multiples of the 256 x 128 tile; several persistent tiles per CTA."""
    ds = synth.generate(synth.scaled(0, n=333, m=1301, t=517, seed=52))
    _, rp, (bp, sp, tp, _) = engine_run(ds, 1, precision=E.PLAIN)
    _, rm, (bm, sm, tm, _) = engine_run(ds, 1, precision=E.MIXED)
    assert np.nanmax(np.abs(tp - tm)) < 1e-3
    np.testing.assert_array_equal(np.isnan(tp), np.isnan(tm))


@pytest.mark.parametrize("variant", ["3", "4"])
@pytest.mark.parametrize("case", ["r1_patterns", "r2_missing", "r1_xrnan"])
def test_cta_pair_gemm_matches_fp64_oracle(case, variant, monkeypatch):
    """The 2-SM (CTA pair) form of the statistics GEMM: same bars as the 1-SM form,
    and the same numbers as the 1-SM form to FP32 rounding (t > 128: narrower trait
    blocks take the 1-SM narrow tiles whatever the variant)."""
    w = synth.scaled(0, **dict(CASES[case], t=150))
    ds = synth.generate(w)
    res, inp, s = oracle_dense(ds, w.r)
    monkeypatch.setenv("OA_TC_VARIANT", variant)
    _, rows3, (b3, se3, t3, r23) = engine_run(ds, w.r, precision=E.MIXED)
    monkeypatch.setenv("OA_TC_VARIANT", "1")
    _, rows1, (b1, se1, t1, r21) = engine_run(ds, w.r, precision=E.MIXED)
    D = res.dense
    ok = ~D.singular
    t_ref = D.tstat[:, :, res.l:][ok]
    dt = np.abs(t3[ok] - t_ref)
    assert np.all(dt <= T_ABS_MIXED + T_REL_MIXED * np.abs(t_ref)), f"max |dt| {dt.max():.3g}"
    np.testing.assert_allclose(t3, t1, rtol=1e-5, atol=1e-5)
    assert rows3.singular == rows1.singular


@pytest.mark.parametrize("variant", ["3", "4"])
def test_cta_pair_gemm_multiple_tiles_and_ragged_edges(variant, monkeypatch):
    """Several 256 x 256 pair tiles per cluster, t and m not multiples of 256."""
    ds = synth.generate(synth.scaled(0, n=333, m=1301, t=517, seed=52))
    monkeypatch.setenv("OA_TC_VARIANT", variant)
    _, r3, (b3, s3, t3, _) = engine_run(ds, 1, precision=E.MIXED)
    monkeypatch.setenv("OA_TC_VARIANT", "1")
    _, r1, (b1, s1, t1, _) = engine_run(ds, 1, precision=E.MIXED)
    np.testing.assert_allclose(t3, t1, rtol=1e-5, atol=1e-5)
    np.testing.assert_array_equal(np.isnan(t3), np.isnan(t1))
    np.testing.assert_array_equal(r3.trait, r1.trait)


@pytest.mark.parametrize("t", [1, 37, 64, 65, 128, 129])
def test_mixed_narrow_trait_tiles(t):
    """Trait blocks of at most 64 / 128 traits run on 64- / 128-column tiles, wider
    ones on 256-column tiles: the same statistics as the FP32 form either side of
    each boundary, several M tiles per CTA, ragged SNP edge."""
    ds = synth.generate(synth.scaled(0, n=517, m=2333, t=t, l=4, miss_mode="patterns", n_patterns=3, seed=60 + t))
    _, rp, (bp, sp, tp, _) = engine_run(ds, 1, precision=E.PLAIN)
    _, rm, (bm, sm, tm, _) = engine_run(ds, 1, precision=E.MIXED)
    assert np.nanmax(np.abs(tp - tm)) < 1e-3
    np.testing.assert_array_equal(np.isnan(tp), np.isnan(tm))
    assert rp.tests == rm.tests == t * 2333
