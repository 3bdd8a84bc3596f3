"""Helpers shared by the parity tests: regenerate golden inputs and compare result sets.

The golden fixtures are outputs of the reference CLI (see
tests/golden/make_golden.py).  Their inputs are regenerated here from the
same seeds and checked against the sha256 digests in the manifest, so the
comparison runs on exactly the bytes the reference read.
"""
from __future__ import annotations

import gzip
import json
import math
import os
import tempfile
from dataclasses import dataclass

import numpy as np

import oa_oracle as O
from golden import make_golden as MG

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def all_runs():
    man = manifest()
    out = []
    for case, entry in sorted(man["cases"].items()):
        for tag, run in sorted(entry["runs"].items()):
            out.append((case, tag))
    return out


def materialise(case: str, where: str):
    """Write the case's inputs under ``where`` and verify their digests."""
    pre, extra = MG.build_inputs(case, where)
    want = manifest()["cases"][case]["inputs"]
    got = MG.input_digests(pre)
    if got != want:
        raise AssertionError(f"{case}: regenerated inputs differ from the golden digests")
    return pre, extra


def settings_for(flags, extra) -> O.Settings:
    s = O.Settings()
    it = iter(flags)
    for f in it:
        if f == "-f":
            s.storePInd = True
        elif f == "-i":
            s.disp_cov = True
        elif f == "-b":
            s.storeBin = True
        elif f == "-n":
            s.r = int(next(it))
        elif f == "-x":
            s.fname_excludelist = next(it).format(**extra)
        elif f in ("-j", "-k", "-l"):
            s.model = {"-j": 1, "-k": 2, "-l": 3}[f]
        elif f in ("-v", "-w"):
            s.fname_interactions = next(it).format(**extra)
            s.multi_interactions = f == "-w"
        elif f in ("-z", "-y"):
            s.model = 4 if f == "-z" else 5
            with open(next(it).format(**extra)) as fh:
                s.factors = tuple(float(v) for v in fh.read().split())
        else:
            raise ValueError(f)
    return s


def golden_rows(case: str, tag: str):
    path = os.path.join(GOLDEN, case, f"{tag}_dis.txt.gz")
    with gzip.open(path, "rt") as f:
        tmp = tempfile.NamedTemporaryFile("w", suffix="_dis.txt", delete=False)
        tmp.write(f.read())
        tmp.close()
    try:
        return O.parse_dis(tmp.name)
    finally:
        os.unlink(tmp.name)


def t_display(minPdisp: float) -> float:
    """|t| at which P(t) = minPdisp on the erfc branch (t >= 1.6)."""
    return math.sqrt(2.0) * _erfcinv(minPdisp)


def _erfcinv(p: float) -> float:
    lo, hi = 0.0, 40.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if math.erfc(mid) > p:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


@dataclass
class Tol:
    t_rel: float
    t_abs: float
    se_rel: float
    r2_abs: float


# Plausibility bound of an FP32 normal-equation solver's answers around exact
# arithmetic (rounding 6e-8 amplified by the conditioning of unscaled
# covariates); the oracle's deviation from every golden run must fall inside it.
REF_TOL = Tol(t_rel=2e-3, t_abs=1e-2, se_rel=2e-4, r2_abs=2e-4)


def noise():
    """The reference's own noise per golden run (tests/golden/noise.json, written by
    tests/golden/measure_noise.py): its 1- vs 8-thread spread and its deviation from FP64."""
    with open(os.path.join(GOLDEN, "noise.json")) as f:
        return json.load(f)


def quirk_noise():
    """The reference's largest deviation from the FP64 oracle per quirk-mode dense test case
    (tests/golden/quirk_noise.json, written by tests/golden/measure_quirk_noise.py)."""
    with open(os.path.join(GOLDEN, "quirk_noise.json")) as f:
        return json.load(f)


def run_tol(case: str, tag: str) -> Tol:
    """Parity bar of the GPU CLI against one golden run: |t - t_ref| <= 1e-4 |t_ref| + delta,
    delta = the reference's own noise on that run (the larger of its thread spread and its
    distance from exact arithmetic beyond 1e-4 |t|) + 1e-4, the plain form's absolute allowance
    against FP64; SE and R2 likewise (the reference's deviation + the plain form's allowance)."""
    m = noise()[case][tag]
    return Tol(t_rel=1e-4, t_abs=max(m["dt_threads"], m["dt_fp64_excess"]) + 1e-4,
               se_rel=m["dse_rel_fp64"] + 1e-4, r2_abs=m["dr2_fp64"] + 1e-4)


def compare_rows(ref_rows, our_rows, tol: Tol, near_boundary):
    """Compare two lists of _dis rows keyed by (Phe, SNP).

    ``near_boundary(phe, snp)`` says whether a row present on one side
    only sits within tolerance of a store/display threshold.  Returns a
    dict of diagnostics; raises AssertionError on a real mismatch.
    """
    rk = {(r["Phe"], r["SNP"]): r for r in ref_rows}
    ok = {(r["Phe"], r["SNP"]): r for r in our_rows}
    if len(rk) != len(ref_rows) or len(ok) != len(our_rows):
        raise AssertionError("duplicate (Phe, SNP) rows")
    only_ref = [k for k in rk if k not in ok]
    only_our = [k for k in ok if k not in rk]
    bad = [k for k in only_ref + only_our if not near_boundary(*k)]
    if bad:
        raise AssertionError(f"{len(bad)} rows differ away from thresholds, e.g. {bad[:5]}")
    worst = dict(t=0.0, se=0.0, r2=0.0)
    for k in rk.keys() & ok.keys():
        a, b = rk[k], ok[k]
        if a["n"] != b["n"] or a["nPct"] != b["nPct"]:
            raise AssertionError(f"{k}: n/nPct {a['n']},{a['nPct']} vs {b['n']},{b['nPct']}")
        dt = abs(a["T"] - b["T"])
        lim = tol.t_rel * abs(a["T"]) + tol.t_abs
        worst["t"] = max(worst["t"], dt / lim)
        if dt > lim:
            raise AssertionError(f"{k}: T {a['T']} vs {b['T']}")
        dse = abs(a["SE"] - b["SE"]) / max(abs(a["SE"]), 1e-30)
        worst["se"] = max(worst["se"], dse / tol.se_rel)
        if dse > tol.se_rel and abs(a["SE"] - b["SE"]) > 1.5e-7:
            raise AssertionError(f"{k}: SE {a['SE']} vs {b['SE']}")
        # B agrees to the same number of standard errors as T
        if abs(a["B"] - b["B"]) > lim * max(a["SE"], b["SE"]) + 1.5e-7:
            raise AssertionError(f"{k}: B {a['B']} vs {b['B']}")
        if abs(a["R2"] - b["R2"]) > tol.r2_abs * max(1.0, abs(a["R2"])):
            raise AssertionError(f"{k}: R2 {a['R2']} vs {b['R2']}")
    # order of the common rows must agree
    order_r = [k for k in (tuple((r["Phe"], r["SNP"])) for r in ref_rows) if k in ok]
    order_o = [k for k in (tuple((r["Phe"], r["SNP"])) for r in our_rows) if k in rk]
    if order_r != order_o:
        raise AssertionError("row order differs")
    return dict(common=len(rk.keys() & ok.keys()), only_ref=len(only_ref), only_our=len(only_our), worst=worst)


def oracle_rows(res: O.Results, inp: O.Inputs, s: O.Settings):
    """The _dis rows the oracle's results print as (numeric fields as float)."""
    disp = O.displayed(res, s)
    names = O.result_names(res, inp, res.l, res.r)
    rows = []
    for i in np.nonzero(disp)[0]:
        rows.append(dict(Phe=names[i][0], SNP=names[i][1], n=int(res.nUsed[i]),
                         nPct=f"{float(res.nUsedPct[i]):.2f}", B=float(res.B[i]),
                         R2=float(np.float32(res.R2[i])), SE=float(res.SE[i]), T=float(res.T[i]),
                         P=None))
    return rows


def boundary_fn(res_dense: O.Results, inp: O.Inputs, s: O.Settings, tol: Tol):
    """near_boundary(phe, snp) from the oracle's dense t of that test's SNP terms."""
    minR2store, minPstore, minT = O.thresholds(s)
    td = t_display(float(np.float32(s.minPdisp)))
    tp = 1.2834  # the 0.5-0.1(4.4-t)t branch reaches P = 0.1 here; displays can flip near it
    yidx = {name: j for j, name in enumerate(inp.y_names)}
    l, r = res_dense.l, res_dense.r
    names = {}
    for i in range(len(inp.xr_names) // r):
        for h in range(r):
            names[" " + inp.xr_names[i * r + h]] = i
        for a in inp.xl_names:
            names[a + ":" + inp.xr_names[i * r]] = i
    D = res_dense.dense

    def near(phe, snp):
        j, i = yidx[phe], names[snp]
        for h in range(l, l + r):
            t = D.tstat[j, i, h]
            lim = 2 * (tol.t_rel * abs(t) + tol.t_abs)
            if min(abs(t - float(minT)), abs(t - td), abs(t - 1.6), abs(t - tp)) <= lim:
                return True
        if abs(D.r2[j, i] - float(minR2store)) <= 2 * tol.r2_abs:
            return True
        return False

    return near


def parse_ibin(raw: bytes):
    import struct
    n, l, r, t, m, nl = struct.unpack_from("<6i", raw, 0)
    disp_cov, store_all = raw[24], raw[25]
    return dict(n=n, l=l, r=r, t=t, m=m, namelength=nl, disp_cov=bool(disp_cov), store_all=bool(store_all))


def ibin_ar_names(raw: bytes):
    """The SNP-term names of a _sto.ibin file (r * m of them, src/AIOwrapper.cpp:693-732)."""
    info = parse_ibin(raw)
    nl = info["namelength"]
    pos = 26 + (info["l"] - 1) * nl
    out = []
    for _ in range(info["r"] * info["m"]):
        out.append(raw[pos:pos + nl].split(b"\0")[0].decode())
        pos += nl
    return out


def parse_dbin(path: str, info: dict):
    """Blocks of a _sto.dbin file (layout: src/AIOwrapper.cpp:1454-1531)."""
    import struct
    raw = open(path, "rb").read()
    pos = 0
    blocks = []
    store_all, disp_cov = info["store_all"], info["disp_cov"]
    if store_all:
        raise NotImplementedError("-f .dbin files carry no block structure")
    while pos < len(raw):
        yidx, cnt, aroff = struct.unpack_from("<3i", raw, pos)
        pos += 12
        rows = []
        for _ in range(cnt):
            nused, r2 = struct.unpack_from("<HH", raw, pos)
            pos += 4
            k = raw[pos]
            pos += 1
            res = []
            for _ in range(k):
                al = None
                if disp_cov:
                    al = raw[pos]
                    pos += 1
                (ar,) = struct.unpack_from("<H", raw, pos)
                pos += 2
                b, se = struct.unpack_from("<ff", raw, pos)
                pos += 8
                res.append((al, ar, b, se))
            rows.append((nused, r2, res))
        blocks.append((yidx, cnt, aroff, rows))
    return blocks


def compare_dbin(ref_path: str, our_path: str, ibin: bytes, exact_rows: bool):
    info = parse_ibin(ibin)
    if info["store_all"]:
        a, b = open(ref_path, "rb").read(), open(our_path, "rb").read()
        assert len(a) == len(b)
        return
    A, B = parse_dbin(ref_path, info), parse_dbin(our_path, info)
    if not exact_rows:
        # boundary rows shift the structure; require the same block headers where counts agree
        assert abs(len(A) - len(B)) <= 1
        return
    assert len(A) == len(B)
    for (ya, ca, oa, ra), (yb, cb, ob, rb) in zip(A, B):
        assert (ya, ca, oa) == (yb, cb, ob)
        for (na, r2a, resa), (nb, r2b, resb) in zip(ra, rb):
            assert na == nb
            assert abs(int(r2a) - int(r2b)) <= 2      # bf16-truncated R2: last bits may differ
            assert len(resa) == len(resb)
            for (ala, ara, ba, sea), (alb, arb, bb, seb) in zip(resa, resb):
                assert (ala, ara) == (alb, arb)
                assert abs(sea - seb) <= 2e-4 * abs(sea) + 1e-7
                assert abs(ba - bb) <= (2e-3 * abs(ba / sea) + 1e-2) * sea + 1e-7
