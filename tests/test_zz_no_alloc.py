"""The zero-allocation entry point, oa_scan_dense_noalloc, against the block
engine and the FP64 oracle.

oa_scan_dense_noalloc serves callers that cannot allocate GPU memory (plug-ins
whose host framework owns the device memory pool, processes whose device
memory was reserved up front): all its intermediates live in one static
device array.  Its dense results must equal the block engine's
(oa_run_snps_device + oa_dense_last with store_all) and the FP64 oracle's
within the plain-form tolerance, on calls in a row with different shapes (the
shared array keeps the previous call's contents, so this also checks that
every call clears what must start at zero) - one of them with observed
phenotypes exactly 0, whose zero sets take their own tables in the array.  A
repeated call must leave the device's free memory (cudaMemGetInfo) unchanged.

This file is collected last on purpose: it needs a GPU and runs after every
other test.
"""
import numpy as np
import pytest

import oa_oracle as O
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


def oracle_dense(ds, r):
    l, n = ds.XL.shape
    inp = O.Inputs(XL=ds.XL, XR=ds.XR, Y=ds.Y, xl_names=ds.xl_names, xr_names=ds.xr_names,
                   y_names=ds.y_names, realN=n, kept=np.arange(n))
    D = O.solve(inp, O.Settings(r=r, storePInd=True), keep_dense=True).dense
    nan = np.float32(np.nan)
    b, se, tt = (np.where(D.singular[:, :, None], nan, a[:, :, l:]).astype(np.float32)
                 for a in (D.beta, D.se, D.tstat))
    return b, se, tt, np.where(D.singular, nan, D.r2).astype(np.float32)


class Device:
    """Device copies of one dataset and output buffers for the entry point."""

    def __init__(self, ds, r):
        import torch
        self.l, self.n = ds.XL.shape
        self.m, self.t, self.r = ds.XR.shape[0] // r, ds.Y.shape[0], r
        dev = torch.device("cuda", 0)
        self.xl = torch.from_numpy(np.ascontiguousarray(ds.XL)).to(dev)
        self.y = torch.from_numpy(np.ascontiguousarray(ds.Y)).to(dev)
        self.xr = torch.from_numpy(np.ascontiguousarray(ds.XR)).to(dev)
        self.beta = torch.empty((self.t, self.m, r), dtype=torch.float32, device=dev)
        self.se = torch.empty_like(self.beta)
        self.tt = torch.empty_like(self.beta)
        self.r2 = torch.empty((self.t, self.m), dtype=torch.float32, device=dev)
        torch.cuda.synchronize()

    def scan(self):
        E.scan_dense_noalloc(self.xl.data_ptr(), self.y.data_ptr(), self.xr.data_ptr(), self.n, self.l, self.r,
                             self.t, self.m, self.beta.data_ptr(), self.se.data_ptr(), self.tt.data_ptr(),
                             self.r2.data_ptr(), 0)

    def results(self):
        return self.beta.cpu().numpy(), self.se.cpu().numpy(), self.tt.cpu().numpy(), self.r2.cpu().numpy()


def noalloc_dense(ds, r):
    d = Device(ds, r)
    d.scan()
    return d.results()


def check_same(a, b, what):
    ba, sa, ta, ra = a
    bb, sb, tb, rb = b
    np.testing.assert_array_equal(np.isnan(ta), np.isnan(tb), err_msg=what)
    ok = ~np.isnan(ta)
    dt = np.abs(ta[ok] - tb[ok])
    assert np.all(dt <= T_REL * np.abs(tb[ok]) + T_ABS), f"{what}: max |dt| {dt.max():.3g}"
    assert np.allclose(sa[ok], sb[ok], rtol=SE_REL, atol=0), what
    assert np.allclose(ba[ok], bb[ok], rtol=0, atol=1e-4 * np.nanmax(np.abs(sb))), what
    okr = ~np.isnan(ra)
    assert np.allclose(ra[okr], rb[okr], rtol=0, atol=1e-5), what


def _yzero(ds, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    for j in range(ds.Y.shape[0]):
        obs = np.nonzero(~np.isnan(ds.Y[j]))[0]
        ds.Y[j, rng.choice(obs, 6, replace=False)] = 0.0
    return ds


def test_noalloc_matches_block_engine_and_oracle_on_calls_in_a_row():
    first = synth.generate(synth.scaled(0, n=500, m=300, t=12, seed=61))
    second = synth.generate(synth.scaled(0, n=640, m=150, t=9, l=4, r=2, miss_mode="patterns", n_patterns=3,
                                         xr_nan_frac=0.01, seed=62))
    third = _yzero(synth.generate(synth.scaled(0, n=400, m=150, t=10, seed=27)), 5)
    for name, ds, r in (("first", first, 1), ("second", second, 2), ("zero phenotypes", third, 1)):
        got = noalloc_dense(ds, r)
        check_same(got, engine_dense(ds, r), name + " vs block engine")
        check_same(got, oracle_dense(ds, r), name + " vs FP64 oracle")


def test_noalloc_repeated_call_allocates_no_device_memory():
    import torch
    ds = synth.generate(synth.scaled(0, n=700, m=260, t=11, l=4, miss_mode="patterns", n_patterns=2, seed=63))
    d = Device(ds, 1)
    d.scan()                       # the first call may load the library's device code and symbol
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    first = d.results()
    d.scan()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes across a call"
    for x, y in zip(first, d.results()):
        np.testing.assert_array_equal(x, y)


def test_noalloc_rejects_collinear_covariates_by_the_engine_rule():
    ds = synth.generate(synth.scaled(0, n=300, m=20, t=3, l=4, seed=64))
    ds.XL[3] = 2.0 * ds.XL[2] - 0.5 * ds.XL[0]          # exactly dependent column
    with pytest.raises(E.OAError) as ei:
        noalloc_dense(ds, 1)
    assert ei.value.status == 3
    with pytest.raises(E.OAError) as ee:
        engine_dense(ds, 1)
    assert ee.value.status == 3


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
