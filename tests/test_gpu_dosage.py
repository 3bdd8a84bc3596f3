"""Dosage models on the GPU (oa_set_column_model): SNPs arrive as genotype-
probability columns and the model columns are formed on the device before the
statistics.  Compared with the FP64 oracle applying the same model on the host
(whose model code is pinned to the reference's own solver by the golden
fixtures); the CLI with -j/-k/-l/-z/-y is compared with the reference's
outputs in test_gpu_parity.py (the r1_dos* golden cases)."""
import numpy as np
import pytest

import oa_oracle as O
from omicabelnomm_b200 import engine as E
from omicabelnomm_b200 import synth
from test_gpu_parity import T_ABS, T_REL

pytestmark = pytest.mark.gpu

MODELS = {  # name: (oracle model, file columns, weights, combine)
    "additive3": (1, 3, (2.0, 1.0, 0.0), True),
    "dominant3": (2, 3, (1.0, 1.0, 0.0), True),
    "recessive3": (3, 3, (1.0, 0.0, 0.0), True),
    "additive2": (1, 2, (2.0, 1.0), True),
    "recessive2": (3, 2, (1.0, 0.0), True),
    "custom_additive2": (5, 2, (0.5, 1.5), True),
    "custom_linear2": (4, 2, (0.5, 1.5), False),
}


def _oracle(ds, model, cols, weights):
    s = O.Settings(r=cols, storePInd=True, model=model, factors=weights if model >= 4 else ())
    XR, names, r = O.column_model(ds.XR, ds.xr_names, s)
    inp = O.Inputs(XL=ds.XL, XR=XR, Y=ds.Y, xl_names=ds.xl_names, xr_names=names, y_names=ds.y_names,
                   realN=ds.XL.shape[1], kept=np.arange(ds.XL.shape[1]), r=r)
    return O.solve(inp, s, keep_dense=True), r


@pytest.mark.parametrize("prec", [E.PLAIN, E.MIXED])
@pytest.mark.parametrize("name", sorted(MODELS))
def test_model_columns_match_oracle(name, prec):
    model, cols, weights, combine = MODELS[name]
    w = synth.scaled(0, n=600, m=300, t=10, l=4, prob_cols=cols, miss_mode="patterns", n_patterns=3,
                     seed=41 + cols)
    ds = synth.generate(w)
    l, n = ds.XL.shape
    m = ds.XR.shape[0] // cols
    res, r = _oracle(ds, model, cols, weights)
    eng = E.Engine(n, l, r, w.t, m, precision=prec, store_all=True, min_t_store=E.t_threshold(0.1),
                   min_r2_store=1e-6)
    eng.set_tuning(chunk_snps=128)                     # several chunks of file columns
    eng.set_covariates(ds.XL)
    eng.set_column_model(cols, weights, combine)
    eng.set_traits(ds.Y)
    eng.enable_dense(True)
    rows = eng.run(ds.XR)
    b, se, tt, r2 = eng.dense(m)
    D = res.dense
    ok = ~D.singular
    t_ref = D.tstat[:, :, l:][ok]
    dt = np.abs(tt[ok] - t_ref)
    lim = (T_REL * np.abs(t_ref) + T_ABS) if prec == E.PLAIN else (1e-3 + 1e-4 * np.abs(t_ref))
    assert np.all(dt <= lim), f"max |dt| {dt.max():.3g}"
    assert rows.tests == w.t * m


def test_device_input_and_model_reset():
    """Device-resident file columns give the host path's numbers; in_cols = 0
    restores plain blocks."""
    import torch
    w = synth.scaled(0, n=500, m=200, t=6, prob_cols=3, seed=47)
    ds = synth.generate(w)
    l, n = ds.XL.shape
    m = ds.XR.shape[0] // 3
    eng = E.Engine(n, l, 1, w.t, m, store_all=True, min_t_store=E.t_threshold(0.1), min_r2_store=1e-6)
    eng.set_covariates(ds.XL)
    eng.set_column_model(3, (2.0, 1.0, 0.0), True)
    eng.set_traits(ds.Y)
    eng.enable_dense(True)
    eng.run(ds.XR)
    host = [a.copy() for a in eng.dense(m)]
    xr = torch.from_numpy(ds.XR).cuda()
    eng.run_device(xr.data_ptr(), m)
    dev = eng.dense(m)
    for a, b in zip(host, dev):
        np.testing.assert_array_equal(a, b)
    # plain blocks again: the combined column computed on the host
    eng.set_column_model(0)
    X = (2.0 * ds.XR[0::3].astype(np.float64) + ds.XR[1::3]).astype(np.float32)
    eng.run(X)
    plain = eng.dense(m)
    np.testing.assert_allclose(plain[2], host[2], rtol=1e-5, atol=1e-5)


def test_model_argument_checks():
    eng = E.Engine(100, 3, 1, 4, 50)
    with pytest.raises(E.OAError):
        eng.set_column_model(2, (1.0, 1.0), False)      # scaled columns need r = 2
    with pytest.raises(E.OAError):
        eng.set_column_model(9, np.ones(9), True)       # at most 8 file columns
    eng.set_column_model(3, (2.0, 1.0, 0.0), True)
    with pytest.raises(E.OAError):
        eng.set_snp_rows(np.arange(100, dtype=np.int32), 200)   # no row subsets with a model


@pytest.mark.parametrize("prec", [E.PLAIN, E.MIXED])
@pytest.mark.parametrize("k,model", [(1, 0), (3, 0), (1, 1)])
def test_interaction_columns_match_oracle(k, model, prec):
    """SNP column x -> [I_1 x, ..., I_k x, x] on the device (r = k + 1), alone and
    after the additive dosage model, with phenotype missingness (the correct
    downdate; the reference's r >= 2 quirk is not reproduced)."""
    cols = 3 if model else 0
    w = synth.scaled(0, n=500, m=120, t=8, l=4, prob_cols=cols, miss_mode="patterns", n_patterns=2, seed=51 + k)
    ds = synth.generate(w)
    l, n = ds.XL.shape
    rng = np.random.Generator(np.random.PCG64(52 + k))
    inter = np.stack([rng.normal(0, 1, n), rng.binomial(1, 0.5, n), rng.uniform(0, 2, n)])[:k].astype(np.float32)
    s = O.Settings(r=cols or 1, storePInd=True, model=model)
    XR, names, r = (O.column_model(ds.XR, ds.xr_names, s) if model else (ds.XR, ds.xr_names, 1))
    XR, names, r = O.interaction_columns(XR, names, r, inter)
    inp = O.Inputs(XL=ds.XL, XR=XR, Y=ds.Y, xl_names=ds.xl_names, xr_names=names, y_names=ds.y_names,
                   realN=n, kept=np.arange(n), r=r)
    res = O.solve(inp, s, keep_dense=True)
    m = ds.XR.shape[0] // (cols or 1)
    eng = E.Engine(n, l, r, w.t, m, precision=prec, store_all=True, min_t_store=E.t_threshold(0.1),
                   min_r2_store=1e-6)
    eng.set_covariates(ds.XL)
    if model:
        eng.set_column_model(cols, (2.0, 1.0, 0.0), True)
    eng.set_interactions(inter, keep=True)
    eng.set_traits(ds.Y)
    eng.enable_dense(True)
    eng.run(ds.XR)
    b, se, tt, r2 = eng.dense(m)
    D = res.dense
    ok = ~D.singular
    t_ref = D.tstat[:, :, l:][ok]
    dt = np.abs(tt[ok] - t_ref)
    lim = (T_REL * np.abs(t_ref) + T_ABS) if prec == E.PLAIN else (1e-3 + 1e-4 * np.abs(t_ref))
    if r >= 2 and prec == E.MIXED:
        lim = lim + 1e-4 * np.abs(t_ref)          # the r >= 2 bar of the mixed form
    assert np.all(dt <= lim), f"max |dt| {dt.max():.3g}"


def test_interaction_argument_checks():
    eng = E.Engine(100, 3, 2, 4, 50)
    with pytest.raises(E.OAError):
        eng.set_interactions(np.ones((2, 100), np.float32), keep=True)   # 2 + 1 != r = 2
    eng.set_interactions(np.ones((1, 100), np.float32), keep=True)
    eng.set_column_model(0)                                              # clears them
    # a combined model may come before its interactions; a block without them is refused
    w = synth.scaled(0, n=100, m=50, t=4, prob_cols=3, seed=5)
    ds = synth.generate(w)
    eng2 = E.Engine(100, w.l, 2, 4, 50)
    eng2.set_covariates(ds.XL)
    eng2.set_column_model(3, (2.0, 1.0, 0.0), True)
    eng2.set_traits(ds.Y)
    with pytest.raises(E.OAError):
        eng2.run(ds.XR)                                                  # r = 2 needs one interaction column
    eng2.set_interactions(np.ones((1, 100), np.float32), keep=True)
    assert eng2.run(ds.XR).tests == 4 * 50


@pytest.mark.parametrize("prec", [E.PLAIN, E.MIXED])
@pytest.mark.parametrize("m,model", [(700, 0), (2, 0), (300, 1)])
def test_multi_interactions_match_oracle(prec, m, model, tmp_path):
    """One analysis per interaction column (-w) through oa_solve: each SNP block goes to the
    device once and is scanned once per column with [I_h x, x]; the rows of all columns are
    merged into the reference's order (700 SNPs: blocks of 166 SNPs x 3 columns and a ragged
    last block; 2 SNPs: fewer SNPs than columns, blocks of one SNP x 3 columns).  With
    phenotype missingness (the correct downdate) against the oracle's restatement.  model = 1:
    three genotype-probability columns per SNP through the additive dosage model first."""
    import golden_util as GU
    from golden import make_golden as MG
    cols = 3 if model else 0
    w = synth.scaled(0, n=500, m=m, t=7, l=4, prob_cols=cols, miss_mode="patterns", n_patterns=3, seed=61)
    ds = synth.generate(w)
    pre = str(tmp_path / "c_")
    synth.write_dataset(ds, pre)
    MG.interaction_file(w.n, 62, pre + "INT", 3)
    s = O.Settings(r=cols or 1, model=model, storePInd=True, fname_interactions=pre + "INT",
                   multi_interactions=True)
    res, inp = O.run_files(pre + "XL", pre + "XR", pre + "Y", s, keep_dense=True)
    out = str(tmp_path / "o")
    o = E.solve(pre + "XL", pre + "XR", pre + "Y", out, r=cols or 1, dosage_model=model, store_all=True,
                precision=prec, interactions=pre + "INT", multi_interactions=True)
    assert o.tests == m * 3 * w.t
    want = GU.oracle_rows(res, inp, s)
    ours = O.parse_dis(out + "_dis.txt")
    assert [(r["Phe"], r["SNP"]) for r in ours] == [(r["Phe"], r["SNP"]) for r in want]
    assert [r["n"] for r in ours] == [r["n"] for r in want]
    t_ref = np.array([r["T"] for r in want])
    dt = np.abs(np.array([r["T"] for r in ours]) - t_ref)
    lim = (T_REL * np.abs(t_ref) + T_ABS + 1e-6) if prec == E.PLAIN else (1e-3 + 2e-4 * np.abs(t_ref))
    assert np.all(dt <= lim), f"max |dt| {dt.max():.3g}"
