"""Failure detection without a GPU fault: every wait of the device pipeline
(the tensor-core GEMMs' stage and accumulator waits, the statistics kernels'
staging waits) is bounded on %globaltimer; when one runs out the kernel sets
an error flag, stops issuing, drains its own copies and MMAs in flight with
the fixed 2 s drain bound, frees its tensor memory and returns.  The host
reads the flag after the block and returns OA_ERR_CUDA with a message.

Here the bound is shortened to 1 ns for one engine (OA_WAIT_LIMIT_NS, read
when an engine is created), so that the waits run out on a small case; the
next engine, created with the default bound, must give correct results in
the same process (the context stays usable)."""
import numpy as np
import pytest

import oa_oracle as O
from omicabelnomm_b200 import engine as E
from omicabelnomm_b200 import synth

pytestmark = pytest.mark.gpu


def _engine(ds, prec):
    l, n = ds.XL.shape
    m, t = ds.XR.shape[0], ds.Y.shape[0]
    eng = E.Engine(n, l, 1, t, m, precision=prec, store_all=True, min_t_store=E.t_threshold(0.1),
                   min_r2_store=1e-6)
    eng.set_covariates(ds.XL)
    eng.set_traits(ds.Y)
    eng.enable_dense(True)
    return eng


@pytest.mark.parametrize("prec", [E.MIXED, E.PLAIN])
def test_wait_timeout_is_reported_and_the_next_engine_is_correct(monkeypatch, prec):
    """Mixed form: t > 128 takes the CTA-pair tensor-core GEMM, whose accumulator and stage
    waits last a whole main loop.  Plain form: its only bounded waits are the statistics
    kernel's staging waits (TMA bulk copies, n % 4 == 0); with 160 KB columns (n = 40,000)
    each copy outlasts the %globaltimer's update step, so the 1 ns bound runs out."""
    if prec == E.MIXED:
        w = dict(n=1024, m=300, t=160)
    else:
        w = dict(n=40000, m=64, t=16)
    ds = synth.generate(synth.scaled(0, l=4, miss_mode="patterns", n_patterns=3, seed=97, **w))
    monkeypatch.setenv("OA_WAIT_LIMIT_NS", "1")
    eng = _engine(ds, prec)
    with pytest.raises(E.OAError) as ei:
        eng.run(ds.XR)
    assert ei.value.status == 2 and "timed out" in str(ei.value)
    eng.close()
    monkeypatch.delenv("OA_WAIT_LIMIT_NS")
    eng = _engine(ds, prec)
    eng.run(ds.XR)
    _, _, tt, _ = eng.dense(ds.XR.shape[0])
    eng.close()
    l, n = ds.XL.shape
    inp = O.Inputs(XL=ds.XL, XR=ds.XR, Y=ds.Y, xl_names=ds.xl_names, xr_names=ds.xr_names, y_names=ds.y_names,
                   realN=n, kept=np.arange(n))
    D = O.solve(inp, O.Settings(r=1, storePInd=True), keep_dense=True).dense
    ok = ~D.singular
    t_ref = D.tstat[:, :, l][ok]
    dt = np.abs(tt[:, :, 0][ok] - t_ref)
    lim = (1e-4 * np.abs(t_ref) + 1e-4) if prec == E.PLAIN else np.full_like(t_ref, 1e-3)
    assert np.all(dt <= lim), f"max |dt| {dt.max():.3g}"
