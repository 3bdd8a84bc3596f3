"""GPU parity of the mixed-precision form (tcgen05 BF16 hi/lo, 3 products,
FP32 accumulate) against the FP64 oracle.  Target: max |dt| <= 1e-3."""
import numpy as np
import pytest

import oa_oracle as O
from omicabelnomm_b200 import engine as E
from omicabelnomm_b200 import synth
from test_gpu_parity import CASES, engine_run, oracle_dense

pytestmark = pytest.mark.gpu

T_ABS_MIXED = 1e-3          # |t_mixed - t_fp64| <= 1e-3
T_REL_MIXED = 0.0


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


def _mixed_dense(ds, r, monkeypatch, fused, **env):
    monkeypatch.setenv("OA_FUSED_SPLIT", "1" if fused else "0")
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    eng, rows, dense = engine_run(ds, r, precision=E.MIXED)
    name = eng.last_kernel_ms()[1]
    eng.close()
    return rows, dense, name


@pytest.mark.parametrize("case", ["narrow64", "narrow128", "pair", "pair_r2", "pair_r4", "uncentred", "variant3"])
def test_fused_split_gemms_give_the_split_copy_bits(case, monkeypatch):
    """The fused forms (FP32 columns split into BF16 hi / lo in shared memory by
    converter warps, no split copy in HBM) give bit-identical statistics to the
    split-copy forms: every trait-tile width (1-SM 64 / 128 columns, CTA pairs),
    r = 1, 2, 4, NaN dosages, centred and uncentred columns, ragged SNP and trait
    edges, several tiles per CTA."""
    from quirk_cases import multicol as _multicol
    env = {}
    r = 1
    if case == "narrow64":
        ds = synth.generate(synth.scaled(0, n=1000, m=1500, t=40, l=4, miss_mode="patterns", n_patterns=3,
                                         xr_nan_frac=0.005, seed=71))
    elif case == "narrow128":
        ds = synth.generate(synth.scaled(0, n=1024, m=1300, t=120, l=5, miss_mode="patterns", n_patterns=4,
                                         xr_nan_frac=0.005, seed=72))
    elif case in ("pair", "variant3"):
        ds = synth.generate(synth.scaled(0, n=996, m=2333, t=517, l=4, miss_mode="patterns", n_patterns=5,
                                         xr_nan_frac=0.005, seed=73))
        if case == "variant3":
            env["OA_TC_VARIANT"] = "3"
    elif case == "pair_r2":
        r = 2
        ds = synth.generate(synth.scaled(0, n=800, m=700, t=300, l=4, r=2, miss_mode="patterns", n_patterns=3,
                                         seed=74))
    elif case == "pair_r4":
        r = 4
        ds = _multicol(4, 75, n=600, m=150, t=270)
    else:
        env["OA_CENTER"] = "0"
        ds = synth.generate(synth.scaled(0, n=1000, m=900, t=300, l=4, miss_mode="patterns", n_patterns=3,
                                         xr_nan_frac=0.005, seed=76))
    rows_f, dense_f, name_f = _mixed_dense(ds, r, monkeypatch, True, **env)
    rows_s, dense_s, name_s = _mixed_dense(ds, r, monkeypatch, False, **env)
    assert name_f.endswith("f") and not name_s.endswith("f"), (name_f, name_s)
    for a, b in zip(dense_f, dense_s):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(rows_f.trait, rows_s.trait)
    np.testing.assert_array_equal(rows_f.snp, rows_s.snp)
    np.testing.assert_array_equal(rows_f.T, rows_s.T)


def test_fused_split_falls_back_when_columns_are_not_16_byte_multiples(monkeypatch):
    """n % 4 != 0: the FP32 columns cannot be TMA tiles; the split copy is used and the
    numbers match the FP64 oracle as before."""
    ds = synth.generate(synth.scaled(0, n=1001, m=600, t=200, seed=77))
    rows, (b, se, tt, r2), name = _mixed_dense(ds, 1, monkeypatch, True)
    assert not name.endswith("f")
    res, _, _ = oracle_dense(ds, 1)
    D = res.dense
    ok = ~D.singular
    t_ref = D.tstat[:, :, res.l:][ok]
    assert np.all(np.abs(tt[ok] - t_ref) <= T_ABS_MIXED + T_REL_MIXED * np.abs(t_ref))
