"""Both forms of the per-SNP statistics stage against the FP64 oracle:
  * "pre":    k_snp_lean (X'X over all rows and over each row set) + one
              GEMM of the SNP block with [Q | Q o m_1 | ... | Q o m_S] +
              k_schur (FP64 Schur complement per pattern and SNP);
  * "gather": k_snp_stats (the same sums with per-row gathers of Q).
The engine picks one by the number of row sets; OA_STATS_PATH forces it.
Cases cover the pre-GEMM tile widths 64, 128 and 256 (several column
tiles), r = 1 and 2, NaN dosages, exact-zero phenotypes and both
precisions."""
import functools

import numpy as np
import pytest

from omicabelnomm_b200 import engine as E
from omicabelnomm_b200 import synth
from test_gpu_parity import CASES, T_ABS, T_REL, _yzero, engine_run, oracle_dense

pytestmark = pytest.mark.gpu

PATH_CASES = {
    "r1_patterns": CASES["r1_patterns"],                       # c2 = 28 -> 64-wide tiles
    "r1_p20": dict(n=900, m=500, t=60, l=4, miss_mode="patterns", n_patterns=20, miss_hi=0.1, seed=61),  # c2 = 84
    "r1_many": dict(n=600, m=300, t=300, l=3, seed=62),         # 300 patterns: c2 = 903, four 256-wide tiles
    "r1_xrnan": CASES["r1_xrnan"],
    "r2_missing": CASES["r2_missing"],
}
T_ABS_MIXED, T_REL_MIXED = 1e-3, 1e-4


@functools.lru_cache(maxsize=None)
def _case(case):
    if case == "r1_yzero":
        ds = _yzero(synth.generate(synth.scaled(0, n=400, m=150, t=10, seed=27)), 5)
        r = 1
    else:
        w = synth.scaled(0, **PATH_CASES[case])
        ds = synth.generate(w)
        r = w.r
    res, _, _ = oracle_dense(ds, r)
    return ds, r, res


@pytest.mark.parametrize("path", ["pre", "gather"])
@pytest.mark.parametrize("prec", [E.PLAIN, E.MIXED])
@pytest.mark.parametrize("case", sorted(PATH_CASES) + ["r1_yzero"])
def test_stats_path_matches_fp64_oracle(case, prec, path, monkeypatch):
    monkeypatch.setenv("OA_STATS_PATH", path)
    ds, r, res = _case(case)
    eng, rows, (b, se, tt, r2) = engine_run(ds, r, precision=prec)
    D = res.dense
    l = res.l
    ok = ~D.singular
    t_ref = D.tstat[:, :, l:][ok]
    dt = np.abs(tt[ok] - t_ref)
    if prec == E.PLAIN:
        lim = T_REL * np.abs(t_ref) + T_ABS
    else:
        lim = T_ABS_MIXED + T_REL_MIXED * np.abs(t_ref)
    assert np.all(dt <= lim), f"max |dt| {dt.max():.3g}, worst ratio {(dt / lim).max():.3g}"
    assert np.allclose(se[ok], D.se[:, :, l:][ok], rtol=1e-4, atol=0)
    assert np.allclose(r2[ok], D.r2[ok], rtol=0, atol=1e-5)
    assert rows.singular == int(D.singular.sum())
    if D.singular.any():
        assert np.all(np.isnan(tt[D.singular]))


def test_paths_agree_on_stored_rows(monkeypatch):
    """Same stored rows (trait, SNP) from both paths on a case with 20 patterns."""
    ds, r, _ = _case("r1_p20")
    got = {}
    for path in ("pre", "gather"):
        monkeypatch.setenv("OA_STATS_PATH", path)
        _, rows, dense = engine_run(ds, r, precision=E.PLAIN)
        got[path] = (rows, dense)
    ra, rb = got["pre"][0], got["gather"][0]
    assert len(ra.trait) == len(rb.trait)
    np.testing.assert_array_equal(ra.trait, rb.trait)
    np.testing.assert_array_equal(ra.snp, rb.snp)
    np.testing.assert_allclose(got["pre"][1][2], got["gather"][1][2], rtol=1e-4, atol=1e-4)


@functools.lru_cache(maxsize=None)
def _long_columns():
    # n_pad = 16,448: one SNP column takes 64 KB of shared memory, so the column-statistics kernel
    # runs 512 threads per CTA by default
    w = synth.scaled(0, n=16448, m=160, t=12, l=4, miss_mode="patterns", n_patterns=3, miss_hi=0.1, seed=64)
    ds = synth.generate(w)
    res, _, _ = oracle_dense(ds, 1)
    return ds, res


@pytest.mark.parametrize("prec", [E.PLAIN, E.MIXED])
def test_column_statistics_thread_counts_match_oracle(prec, monkeypatch):
    """Long columns: the 512-thread launch (default at this n) and the 256-thread launch
    (OA_LEAN_THREADS=256) both match the FP64 oracle, and each other within FP32 rounding."""
    ds, res = _long_columns()
    D = res.dense
    ok = ~D.singular
    t_ref = D.tstat[:, :, res.l:][ok]
    got = {}
    for threads in ("512", "256"):
        monkeypatch.setenv("OA_LEAN_THREADS", threads)
        monkeypatch.setenv("OA_STATS_PATH", "pre")
        _, _, (_, _, tt, _) = engine_run(ds, 1, precision=prec)
        got[threads] = tt[ok]
        dt = np.abs(tt[ok] - t_ref)
        lim = (T_REL * np.abs(t_ref) + T_ABS) if prec == E.PLAIN else np.full_like(t_ref, 1e-3)
        assert np.all(dt <= lim), f"{threads} threads: max |dt| {dt.max():.3g}"
    assert np.all(np.abs(got["512"] - got["256"]) <= 1e-4 * np.abs(got["256"]) + 1e-4)
