"""The zero-allocation entry point, oa_scan_dense_noalloc, against the block engine.

oa_scan_dense_noalloc serves callers that cannot allocate GPU memory (code
recording a CUDA graph, plug-ins whose host framework owns the memory pool,
processes with device memory reserved up front): all its intermediates live
in one static device array.  Its dense results must equal the block engine's
(oa_run_snps_device + oa_dense_last with store_all) within the plain-form
tolerance, on two calls in a row with different shapes (the shared array
keeps the previous call's contents, so this also checks that every call
clears what must start at zero).

This file is collected last on purpose: it needs a GPU and runs after every
other test.
"""
import numpy as np
import pytest

from omicabelnomm_b200 import engine as E
from omicabelnomm_b200 import synth

pytestmark = pytest.mark.gpu

T_REL, T_ABS, SE_REL = 1e-4, 1e-4, 1e-4     # the plain form's tolerances (tests/test_gpu_parity.py)


def engine_dense(ds, r):
    l, n = ds.XL.shape
    m, t = ds.XR.shape[0] // r, ds.Y.shape[0]
    eng = E.Engine(n, l, r, t, m, store_all=True, min_t_store=E.t_threshold(0.1), min_r2_store=1e-6)
    eng.set_covariates(ds.XL)
    eng.set_traits(ds.Y)
    eng.enable_dense(True)
    eng.run(ds.XR)
    out = eng.dense(m)
    eng.close()
    return out


def noalloc_dense(ds, r):
    import torch
    l, n = ds.XL.shape
    m, t = ds.XR.shape[0] // r, ds.Y.shape[0]
    dev = torch.device("cuda", 0)
    xl = torch.from_numpy(np.ascontiguousarray(ds.XL)).to(dev)
    y = torch.from_numpy(np.ascontiguousarray(ds.Y)).to(dev)
    xr = torch.from_numpy(np.ascontiguousarray(ds.XR)).to(dev)
    beta = torch.empty((t, m, r), dtype=torch.float32, device=dev)
    se = torch.empty_like(beta)
    tt = torch.empty_like(beta)
    r2 = torch.empty((t, m), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    E.scan_dense_noalloc(xl.data_ptr(), y.data_ptr(), xr.data_ptr(), n, l, r, t, m, beta.data_ptr(),
                         se.data_ptr(), tt.data_ptr(), r2.data_ptr(), 0)
    return beta.cpu().numpy(), se.cpu().numpy(), tt.cpu().numpy(), r2.cpu().numpy()


def check_same(a, b):
    ba, sa, ta, ra = a
    bb, sb, tb, rb = b
    np.testing.assert_array_equal(np.isnan(ta), np.isnan(tb))
    ok = ~np.isnan(ta)
    assert np.all(np.abs(ta[ok] - tb[ok]) <= T_REL * np.abs(ta[ok]) + T_ABS)
    assert np.allclose(sa[ok], sb[ok], rtol=SE_REL, atol=0)
    assert np.allclose(ba[ok], bb[ok], rtol=0, atol=1e-4 * np.nanmax(np.abs(sa)))
    okr = ~np.isnan(ra)
    assert np.allclose(ra[okr], rb[okr], rtol=0, atol=1e-5)


def test_noalloc_matches_block_engine_on_two_calls():
    first = synth.generate(synth.scaled(0, n=500, m=300, t=12, seed=61))
    second = synth.generate(synth.scaled(0, n=640, m=150, t=9, l=4, r=2, miss_mode="patterns", n_patterns=3,
                                         xr_nan_frac=0.01, seed=62))
    for ds, r in ((first, 1), (second, 2)):
        check_same(noalloc_dense(ds, r), engine_dense(ds, r))


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    n, l, r, t, m = 40000, 3, 1, 2000, 64          # 4*n*t alone exceeds the 64 MiB array
    dev = torch.device("cuda", 0)
    xl = torch.zeros((l, n), device=dev)
    y = torch.zeros((t, n), device=dev)
    xr = torch.zeros((m, n), device=dev)
    out = torch.empty((t, m), device=dev)
    with pytest.raises(E.OAError) as ei:
        E.scan_dense_noalloc(xl.data_ptr(), y.data_ptr(), xr.data_ptr(), n, l, r, t, m, out.data_ptr(),
                             out.data_ptr(), out.data_ptr(), out.data_ptr(), 0)
    assert ei.value.status == 7 and "scratch" in str(ei.value)
