"""GPU parity: the CUDA engine through the C ABI against the FP64 oracle and
against the reference's own outputs (golden fixtures).  Needs a B200."""
import os
import subprocess

import numpy as np
import pytest

import golden_util as GU
import oa_oracle as O
import quirk_cases as QC
from omicabelnomm_b200 import engine as E
from omicabelnomm_b200 import synth

pytestmark = pytest.mark.gpu

# Plain FP32 form vs the FP64 oracle: |dt| <= T_REL*|t| + T_ABS, SE within SE_REL.
T_REL, T_ABS, SE_REL = 1e-4, 1e-4, 1e-4


def oracle_dense(ds, r, disp_cov=False):
    inp = O.Inputs(XL=ds.XL, XR=ds.XR, Y=ds.Y, xl_names=ds.xl_names, xr_names=ds.xr_names,
                   y_names=ds.y_names, realN=ds.XL.shape[1], kept=np.arange(ds.XL.shape[1]))
    s = O.Settings(r=r, storePInd=True, disp_cov=disp_cov)
    return O.solve(inp, s, keep_dense=True), inp, s


def engine_run(ds, r, precision=E.PLAIN, store_all=True, disp_cov=False, max_snps=None):
    l, n = ds.XL.shape
    m = ds.XR.shape[0] // r
    t = ds.Y.shape[0]
    eng = E.Engine(n, l, r, t, max_snps or m, precision=precision, store_all=store_all, disp_cov=disp_cov,
                   min_t_store=E.t_threshold(0.1), min_r2_store=1e-6)
    eng.set_covariates(ds.XL)
    eng.set_traits(ds.Y)
    eng.enable_dense(True)
    rows = eng.run(ds.XR)
    dense = eng.dense(m)
    return eng, rows, dense


CASES = {
    "r1_uniform": dict(n=400, m=300, t=20, seed=21),
    "r1_patterns": dict(n=700, m=650, t=40, l=4, miss_mode="patterns", n_patterns=6, miss_hi=0.1, seed=22),
    "r1_xrnan": dict(n=500, m=200, t=12, xr_nan_frac=0.02, seed=23),
    "r1_collinear": dict(n=1500, m=300, t=10, l=5, collinear=True, low_maf_frac=0.05, maf_lo=0.01, seed=24),
    "r2_complete": dict(n=500, m=120, t=10, l=4, r=2, miss_mode="none", seed=25),
    "r2_missing": dict(n=600, m=120, t=16, l=5, r=2, miss_mode="patterns", n_patterns=4, miss_hi=0.15,
                       seed=26),
}


def _yzero(ds, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    for j in range(ds.Y.shape[0]):
        obs = np.nonzero(~np.isnan(ds.Y[j]))[0]
        ds.Y[j, rng.choice(obs, 6, replace=False)] = 0.0
    return ds


@pytest.mark.parametrize("case", sorted(CASES) + ["r1_yzero"])
def test_dense_matches_fp64_oracle(case):
    if case == "r1_yzero":
        ds = _yzero(synth.generate(synth.scaled(0, n=400, m=150, t=10, seed=27)), 5)
        r = 1
    else:
        w = synth.scaled(0, **CASES[case])
        ds = synth.generate(w)
        r = w.r
    res, inp, s = oracle_dense(ds, r)
    eng, rows, (b, se, tt, r2) = engine_run(ds, r)
    D = res.dense
    l = res.l
    ok = ~D.singular
    t_ref = D.tstat[:, :, l:][ok]
    dt = np.abs(tt[ok] - t_ref)
    lim = T_REL * np.abs(t_ref) + T_ABS
    assert np.all(dt <= lim), f"max |dt| {dt.max():.3g}, worst ratio {(dt / lim).max():.3g}"
    assert np.allclose(se[ok], D.se[:, :, l:][ok], rtol=SE_REL, atol=0)
    assert np.allclose(b[ok], D.beta[:, :, l:][ok], rtol=0, atol=1e-4 * np.abs(D.se[:, :, l:][ok]).max())
    assert np.allclose(r2[ok], D.r2[ok], rtol=0, atol=1e-5)
    # every test stored with -f semantics, in (trait, SNP) order
    m = ds.XR.shape[0] // r
    assert rows.tests == ds.Y.shape[0] * m
    key = rows.trait.astype(np.int64) * m + rows.snp
    assert np.all(np.diff(key) > 0)
    assert rows.singular == int(D.singular.sum())


def test_stored_rows_match_oracle_filters():
    ds = synth.generate(synth.scaled(0, n=600, m=400, t=25, seed=31))
    inp = O.Inputs(XL=ds.XL, XR=ds.XR, Y=ds.Y, xl_names=ds.xl_names, xr_names=ds.xr_names,
                   y_names=ds.y_names, realN=ds.XL.shape[1], kept=np.arange(ds.XL.shape[1]))
    s = O.Settings()
    res = O.solve(inp, s, keep_dense=True)
    minR2, _, minT = O.thresholds(s)
    eng = E.Engine(600, 3, 1, 25, 400, min_t_store=float(minT), min_r2_store=float(minR2))
    eng.set_covariates(ds.XL)
    eng.set_traits(ds.Y)
    rows = eng.run(ds.XR)
    got = set(zip(rows.trait.tolist(), rows.snp.tolist()))
    want = set(zip(res.trait.tolist(), res.snp.tolist()))
    diff = got ^ want
    tl = res.dense.tstat[:, :, res.l]
    for j, i in diff:   # only tests sitting on the threshold may differ
        assert abs(tl[j, i] - float(minT)) < 1e-3, (j, i, tl[j, i])
    assert len(diff) <= 2


def test_chunked_block_equals_single_block(monkeypatch):
    """Results do not depend on how a SNP block is split into device chunks."""
    ds = synth.generate(synth.scaled(0, n=300, m=900, t=9, seed=41))
    _, rows_a, dense_a = engine_run(ds, 1)
    monkeypatch.setenv("OA_CHUNK_SNPS", "128")
    _, rows_b, dense_b = engine_run(ds, 1)
    for x, y in zip(dense_a, dense_b):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(rows_a.snp, rows_b.snp)


def _same_count_patterns(seed=91, n=500, m=120, t=16, l=4, miss=25, zeros=5):
    """Traits in four missingness patterns and four zero sets, all patterns with
    the same number of NaN rows and all zero sets with the same number of rows:
    grouping on row counts alone would merge them."""
    ds = synth.generate(synth.scaled(0, n=n, m=m, t=t, l=l, miss_mode="none", seed=seed))
    rng = np.random.Generator(np.random.PCG64(seed))
    pats = [rng.choice(n, miss, replace=False) for _ in range(4)]
    zsets = [rng.choice(n, zeros, replace=False) for _ in range(4)]
    for j in range(t):
        ds.Y[j, zsets[(j // 4) % 4]] = 0.0
        ds.Y[j, pats[j % 4]] = np.nan                   # NaN last: a zero row may become missing
    return ds


def test_trait_grouping_is_exact_under_hash_collisions(monkeypatch):
    """Traits are grouped by (row count, two hash sums) of their NaN rows and
    of their observed exact-zero rows, then checked row by row on the device;
    a collision makes the engine regroup on the exact row masks.  With the
    hash sums cut to 0 bits (every pattern of equal count collides) the
    results must equal those of the full hashes bit for bit, and the oracle's."""
    ds = _same_count_patterns()
    _, rows_a, dense_a = engine_run(ds, 1)
    monkeypatch.setenv("OA_TEST_HASH_BITS", "0")
    _, rows_b, dense_b = engine_run(ds, 1)
    for x, y in zip(dense_a, dense_b):
        np.testing.assert_array_equal(x, y)
    res, _, _ = oracle_dense(ds, 1)
    D = res.dense
    ok = ~D.singular
    t_ref = D.tstat[:, :, res.l:][ok]
    dt = np.abs(dense_b[2][ok] - t_ref)
    assert np.all(dt <= T_REL * np.abs(t_ref) + T_ABS), dt.max()


# ---------------------------------------------------------------------------
# the CLI against the reference's own outputs
# ---------------------------------------------------------------------------
# golden runs where the reference's r >= 2 downdate applies (r = 2 with phenotype missingness)
QUIRK_RUNS = {("r2_missing", "nf"), ("r1_dosf", "nz"), ("r3_missing", "nf")}


def run_cli(pre, extra, flags, out, precision="plain"):
    args = [f.format(**extra) for f in flags]
    cmd = [E.CLI_PATH, "-c", pre + "XL", "-g", pre + "XR", "-p", pre + "Y", "-o", out,
           "--precision", precision] + args
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    return int(p.stdout.split("Number of Significant Results:")[1].split()[0])


@pytest.mark.parametrize("case,tag", GU.all_runs())
def test_cli_matches_reference_outputs(case, tag, tmp_path):
    pre, extra = GU.materialise(case, str(tmp_path))
    run = GU.manifest()["cases"][case]["runs"][tag]
    quirk = (case, tag) in QUIRK_RUNS
    out = str(tmp_path / "gpu")
    sig = run_cli(pre, extra, run["flags"] + (["--quirk-r2"] if quirk else []), out)
    s = GU.settings_for([f for f in run["flags"]], extra)
    s.quirk_r2 = quirk
    res, inp = O.run_files(pre + "XL", pre + "XR", pre + "Y", s, keep_dense=True)
    tol = GU.run_tol(case, tag)
    near = GU.boundary_fn(res, inp, s, tol)
    ref = GU.golden_rows(case, tag)
    ours = O.parse_dis(out + "_dis.txt")
    info = GU.compare_rows(ref, ours, tol, near)
    assert abs(sig - run["significant"]) <= max(2, 0.01 * run["significant"])
    if "-b" in run["flags"] and "-w" in run["flags"]:
        # the reference's .ibin name list for -w reads past its name table (not kept as a
        # fixture): the header must give the run's shape and the names those of the text output
        with open(out + "_sto.ibin", "rb") as f:
            got = f.read()
        hdr = GU.parse_ibin(got)
        pairs = inp.XR.shape[0] // 2
        assert (hdr["n"], hdr["l"], hdr["r"], hdr["t"], hdr["m"]) == (
            inp.XL.shape[1], inp.XL.shape[0], 2, inp.Y.shape[0], pairs)
        assert GU.ibin_ar_names(got) == inp.xr_names
        GU.compare_dbin(os.path.join(GU.GOLDEN, case, f"{tag}_sto.dbin"), out + "_sto.dbin", got,
                        exact_rows=(info["only_ref"] == 0 and info["only_our"] == 0
                                    and sig == run["significant"]))
    elif "-b" in run["flags"]:
        with open(os.path.join(GU.GOLDEN, case, f"{tag}_sto.ibin"), "rb") as f:
            want = f.read()
        with open(out + "_sto.ibin", "rb") as f:
            got = f.read()
        assert got == want, "the .ibin header/names must be byte-identical"
        GU.compare_dbin(os.path.join(GU.GOLDEN, case, f"{tag}_sto.dbin"), out + "_sto.dbin", want,
                        exact_rows=(info["only_ref"] == 0 and info["only_our"] == 0
                                    and sig == run["significant"]))


def test_device_path_graph_replay_matches_uncaptured(monkeypatch):
    """The device-resident scan captured as a CUDA graph gives the uncaptured results, call after call."""
    import torch
    ds = synth.generate(synth.scaled(0, n=512, m=700, t=40, l=4, miss_mode="patterns", n_patterns=5, seed=71))
    l, n = ds.XL.shape
    m, t = ds.XR.shape[0], ds.Y.shape[0]
    dev = torch.device("cuda", 0)
    xr = torch.from_numpy(ds.XR).to(dev)
    y = torch.from_numpy(ds.Y).to(dev)
    monkeypatch.setenv("OA_CHUNK_SNPS", "256")       # several chunks in the graph
    outs = {}
    for graphs in ("0", "1"):
        monkeypatch.setenv("OA_GRAPHS", graphs)
        for prec in (E.PLAIN, E.MIXED):
            eng = E.Engine(n, l, 1, t, m, precision=prec, min_t_store=E.t_threshold(0.1), min_r2_store=1e-6)
            eng.set_covariates(ds.XL)
            eng.set_traits_device(y.data_ptr(), t)
            eng.enable_dense(True)
            counts = []
            for _ in range(3):                        # uncaptured, captured, replayed
                r = eng.run_device(xr.data_ptr(), m)
                counts.append((r.count, r.singular))
                dense = eng.dense(m)
            assert counts[0] == counts[1] == counts[2]
            outs[(graphs, prec)] = (counts[0], dense)
            eng.close()
    for prec in (E.PLAIN, E.MIXED):
        (c0, d0), (c1, d1) = outs[("0", prec)], outs[("1", prec)]
        assert c0 == c1
        for a, b in zip(d0, d1):
            np.testing.assert_array_equal(a, b)


def _flag_case():
    """Planted singular tests: a monomorphic SNP, a SNP equal to the sex
    covariate, and a SNP that varies only on the rows one missingness pattern
    lacks (singular for the traits of that pattern alone)."""
    ds = synth.generate(synth.scaled(0, n=800, m=120, t=30, l=4, miss_mode="patterns", n_patterns=4,
                                     miss_hi=0.12, seed=72))
    rng = np.random.Generator(np.random.PCG64(73))
    ds.XR[3] = 1.0
    ds.XR[7] = ds.XL[1]
    miss0 = np.isnan(ds.Y[0])
    x = np.zeros(ds.XR.shape[1], np.float32)
    x[miss0] = np.round(rng.uniform(0.0, 2.0, int(miss0.sum())), 3)
    ds.XR[11] = x
    return ds


@pytest.mark.parametrize("prec", [E.PLAIN, E.MIXED])
@pytest.mark.parametrize("stats_path", [1, 2])
def test_dense_flags_match_oracle_masks(prec, stats_path):
    """Per-test status bits against the FP64 oracle: singular and RSS bits
    element by element; the R2-filter and stored bits too, except for tests
    whose R2 or largest |t| sits within rounding of its threshold."""
    ds = _flag_case()
    l, n = ds.XL.shape
    m, t = ds.XR.shape[0], ds.Y.shape[0]
    res, _, _ = oracle_dense(ds, 1)
    D = res.dense
    min_t = E.t_threshold(0.05)
    min_r2 = float(np.float32(np.median(D.r2[~D.singular])))
    eng = E.Engine(n, l, 1, t, m, precision=prec, min_t_store=min_t, min_r2_store=min_r2)
    eng.set_covariates(ds.XL)
    eng.set_traits(ds.Y)
    eng.set_tuning(stats_path=stats_path)
    eng.enable_dense(True)
    rows = eng.run(ds.XR)
    f = eng.dense_flags(m)
    sing = D.singular
    assert sing[:, 3].all() and sing[:, 7].all() and sing[0, 11]
    assert not sing[:, 11].all(), "the pattern-only SNP must stay regular for other patterns"
    np.testing.assert_array_equal((f & E.TEST_SINGULAR) != 0, sing)
    np.testing.assert_array_equal((f & E.TEST_RSS) != 0, (D.rss <= 0) & ~sing)
    assert rows.singular == int(sing.sum())
    reg = ~sing & (D.rss > 0)
    want_r2 = reg & ~(D.r2 > min_r2)
    tmax = D.tstat[:, :, l]
    want_st = reg & (D.r2 > min_r2) & (tmax > min_t)
    near = (np.abs(D.r2 - min_r2) < 1e-5) | (np.abs(tmax - min_t) < 1e-3)
    got_r2 = (f & E.TEST_R2) != 0
    got_st = (f & E.TEST_STORED) != 0
    assert not np.any((got_r2 != want_r2) & ~near)
    assert not np.any((got_st != want_st) & ~near)
    # a test has a row exactly when its STORED bit is set
    stored = set(zip(*np.nonzero(got_st)))
    assert stored == set(zip(rows.trait.tolist(), rows.snp.tolist()))


@pytest.mark.parametrize("prec", [E.PLAIN, E.MIXED])
@pytest.mark.parametrize("case", QC.CASES)
def test_quirk_r2_matches_oracle_quirk(case, prec):
    """The reference's r >= 2 downdate reproduced on the device (quirk mode) against the
    oracle's restatement of it: dense t, SE, R2 and the singular set; also with observed
    zero phenotypes (zero sets), with r > l (the SNP-block downdate quirk) and with r = 3
    and 5 (zero padding columns in the kernels).

    The quirk's downdate can leave a system far from positive definite, and its SE and R2
    then carry rounding amplified by the condition number - the reference's own FP32
    answers too: tests/golden/quirk_noise.json holds, per case, the reference's largest
    deviation from the FP64 oracle (tests/golden/measure_quirk_noise.py).  Bars: t as the
    plain form's (relative to the system's largest |t|) or the mixed form's; SE and R2
    within twice the reference's deviation, scaled for the mixed form by 2^7 (the ratio of
    its split's unit roundoff, 2^-17, to FP32's), and never below 1e-3 (SE, relative) and
    1e-4 (R2, relative to max(|R2|, 1))."""
    r, ds = QC.build(case)
    l, n = ds.XL.shape
    m, t = ds.XR.shape[0] // r, ds.Y.shape[0]
    inp = O.Inputs(XL=ds.XL, XR=ds.XR, Y=ds.Y, xl_names=ds.xl_names, xr_names=ds.xr_names,
                   y_names=ds.y_names, realN=n, kept=np.arange(n))
    D = O.solve(inp, O.Settings(r=r, storePInd=True, quirk_r2=True), keep_dense=True).dense
    Dc = O.solve(inp, O.Settings(r=r, storePInd=True), keep_dense=True).dense
    eng = E.Engine(n, l, r, t, m, precision=prec, store_all=True, quirk_r2=True,
                   min_t_store=E.t_threshold(0.1), min_r2_store=1e-6)
    eng.set_covariates(ds.XL)
    eng.set_traits(ds.Y)
    eng.enable_dense(True)
    rows = eng.run(ds.XR)
    b, se, tt, r2 = eng.dense(m)
    ok = ~D.singular
    t_ref = D.tstat[:, :, l:][ok]
    dt = np.abs(tt[ok] - t_ref)
    t_sys = np.broadcast_to(np.abs(t_ref).max(axis=1, keepdims=True), t_ref.shape)
    lim = (T_REL * t_sys + T_ABS) if prec == E.PLAIN else (1e-3 + 5e-4 * t_sys)
    assert rows.singular == int(D.singular.sum()), (rows.singular, int(D.singular.sum()))
    assert np.all(dt <= lim), f"max |dt| {dt.max():.3g}"
    noise = GU.quirk_noise()[case]
    scale = 2.0 * (1.0 if prec == E.PLAIN else 2.0 ** 7)
    dse = np.abs(se[ok] - D.se[:, :, l:][ok]) / np.abs(D.se[:, :, l:][ok])
    q = np.unravel_index(np.argmax(dse), dse.shape)
    assert dse.max() <= max(1e-3, scale * noise["dse_rel"]), (float(dse.max()), float(se[ok][q]),
                                                               float(D.se[:, :, l:][ok][q]))
    dr2 = np.abs(r2[ok] - D.r2[ok]) / np.maximum(np.abs(D.r2[ok]), 1.0)
    assert dr2.max() <= max(1e-4, scale * noise["dr2"]), (float(dr2.max()), float(r2[ok][np.argmax(dr2)]),
                                                          float(D.r2[ok][np.argmax(dr2)]))
    # the quirk matters here: its answers are not the corrected ones
    assert np.abs(D.tstat[:, :, l:] - Dc.tstat[:, :, l:])[ok].max() > 1e-2


@pytest.mark.parametrize("prec", [E.PLAIN, E.MIXED])
@pytest.mark.parametrize("r", [3, 5, 6, 8])
def test_dense_more_columns_per_snp_match_fp64_oracle(r, prec):
    """r = 3, 5, 6 (kernels with 4 or 8 columns per SNP, zero columns added on the device)
    and r = 8, with missingness patterns, against the FP64 oracle; plain bars for the
    plain form, the r >= 2 mixed bars for the mixed form."""
    ds = QC.multicol(r, 80 + r, m=24, t=10)
    res, _, _ = oracle_dense(ds, r)
    eng, rows, (b, se, tt, r2) = engine_run(ds, r, precision=prec)
    D = res.dense
    l = res.l
    ok = ~D.singular
    t_ref = D.tstat[:, :, l:][ok]
    dt = np.abs(tt[ok] - t_ref)
    t_sys = np.broadcast_to(np.abs(t_ref).max(axis=1, keepdims=True), t_ref.shape)
    lim = (T_REL * t_sys + T_ABS) if prec == E.PLAIN else (1e-3 + 1e-4 * t_sys)
    assert np.all(dt <= lim), f"max |dt| {dt.max():.3g}"
    assert np.allclose(se[ok], D.se[:, :, l:][ok], rtol=SE_REL if prec == E.PLAIN else 1e-3, atol=0)
    assert tt.shape == (ds.Y.shape[0], ds.XR.shape[0] // r, r)
    assert rows.singular == int(D.singular.sum())
    # stored rows carry the r SNP terms (p = l + r coefficients per row)
    assert rows.B.shape[1] == l + r
