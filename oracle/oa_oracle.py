"""FP64 CPU oracle for the OmicABELnoMM association engine.  TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only the test suite, the
smoke check and the CPU-baseline leg of the benchmark may import it.  It
restates, in float64 numpy, what the reference computes on its hot path
(``Algorithm::partialNEQ_Blocked_STL_MD``, src/Algorithm.cpp:322-886) and
the reader semantics that decide which individuals take part
(src/AIOwrapper.cpp).  It is pinned against the reference itself: the
golden fixtures under tests/golden/ were produced by the reference CLI
compiled from its own sources (oracle/Makefile), and the CPU tests check
this restatement against them.

Every step cites the reference line it follows.  The restatement solves
each system the way the reference does (full normal equations of the
corrected p x p matrix S, one solve per SNP x trait), not the way the GPU
engine does (covariate projection and Schur complements), so agreement
between the two is an independent check.

Reference semantics reproduced on purpose:

* y NaN -> 0 and the trait's missing rows are downdated from X'X
  (src/Utility.cpp:329-378, src/Algorithm.cpp:1324-1399);
* XR NaN -> mean of the column's non-NaN entries (src/Utility.cpp:302-326);
* SE uses the diagonal of the *uncorrected* (all-rows) inverse times
  (n - miss)/n (src/Algorithm.cpp:646-678, 1034-1134);
* RSS skips rows whose (NaN-zeroed) y is exactly 0 (src/Algorithm.cpp:1013-1020);
* R2 = 1 - (RSS/(n_corr-1)) / (SST/(n-1)), SST over the observed rows
  (src/Algorithm.cpp:1092, 1222-1251);
* P = 0.5 - 0.1*(4.4-t)*t for t < 1.6, else erfc(t/sqrt 2) (src/Algorithm.cpp:1159-1167);
* thresholds, loop order h = p-1 .. start_h and the result/row filters
  (src/Algorithm.cpp:338-342, 359, 1119-1203; src/AIOwrapper.cpp:1494);
* output order Y block -> SNP block -> trait -> SNP -> h descending, with
  tb = min(t, 1000), mb = min(m, 500) (src/AIOwrapper.cpp:212-216); with one
  analysis per interaction column (-w) the blocks are max(1, mb // k) * k
  (SNP, column) pairs (src/AIOwrapper.cpp:441-452).

``quirk_r2=True`` additionally reproduces the reference's r >= 2 downdate
bug (src/Algorithm.cpp:1300 and 1390-1396); the default computes the
correct observed-rows Gram matrix.
"""
from __future__ import annotations

import math
import os
import struct
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

ONE_OVER_SQRT2 = 0.7071067811865475244008443621048490392848359376884740


# ----------------------------------------------------------------------------
# settings and thresholds
# ----------------------------------------------------------------------------
@dataclass
class Settings:
    """The fields of ``struct Settings`` (src/Definitions.h:168-219) that the path reads.

    Defaults follow ``Algorithm::applyDefaultParams`` (src/Algorithm.cpp:277-311).
    """
    r: int = 1
    minPdisp: float = 0.05
    minPstore: float = 0.1
    minR2disp: float = 0.000001
    minR2store: float = 0.00001
    storeBin: bool = False       # -b
    storePInd: bool = False      # -f
    disp_cov: bool = False       # -i
    fname_excludelist: str = ""  # -x
    quirk_r2: bool = False
    model: int = 0               # dosage model: 0 none, 1 additive (-j), 2 dominant (-k), 3 recessive (-l),
                                 # 4 custom linear (-z), 5 custom additive (-y); r is then the file's
                                 # columns per SNP (-n)
    factors: tuple = ()          # -z / -y factors, one per file column of a SNP
    fname_interactions: str = "" # -v: single-set interactions (the SNP column is kept)
    multi_interactions: bool = False  # -w: one analysis per interaction column (with fname_interactions)


# Factors of the fixed dosage models on genotype probabilities (AA, AB, BB)
# (src/AIOwrapper.cpp:268-321); a zero factor drops its column, which the
# reference does not read.
MODEL_FACTORS = {1: (2.0, 1.0, 0.0), 2: (1.0, 1.0, 0.0), 3: (1.0, 0.0, 0.0)}


def column_model(XR: np.ndarray, names: List[str], s: "Settings"):
    """The reference's dosage models (src/AIOwrapper.cpp:257-340, 1213-1275):
    (m*fileR, n) file columns -> (m*r, n) model columns, their names and r.
    Combined models give one column per SNP, named after its first file column."""
    fr = s.r
    m = XR.shape[0] // fr
    if s.model in MODEL_FACTORS:
        if fr not in (2, 3):
            raise ValueError("the fixed dosage models take 2 or 3 columns per SNP")
        w, combine = MODEL_FACTORS[s.model][:fr], True
    elif s.model in (4, 5):
        if len(s.factors) != fr:
            raise ValueError("one factor per file column")
        w, combine = tuple(float(f) for f in s.factors), s.model == 5
    else:
        raise ValueError(f"dosage model {s.model}")
    cols = XR.reshape(m, fr, -1).astype(np.float64)
    if combine:
        out = np.zeros((m, cols.shape[2]))
        for c, wc in enumerate(w):
            if wc != 0.0:
                out += wc * cols[:, c]
        return out.astype(np.float32), [names[i * fr] for i in range(m)], 1
    out = cols * np.asarray(w)[None, :, None]
    return out.reshape(m * fr, -1).astype(np.float32), list(names), fr


def interaction_columns(XR: np.ndarray, names: List[str], r: int, inter: np.ndarray):
    """Single-set interactions (src/AIOwrapper.cpp:808-840, names :566-612): each
    SNP column x -> [I_1 x, ..., I_k x, x], named "I<h>x<name>" and <name>."""
    if r != 1:
        raise ValueError("interactions need one column per SNP")
    k, m = inter.shape[0], XR.shape[0]
    out = np.empty((m * (k + 1), XR.shape[1]), dtype=np.float32)
    out_names = []
    for i in range(m):
        for h in range(k):
            out[i * (k + 1) + h] = inter[h] * XR[i]
            out_names.append(f"I{h + 1}x{names[i]}")
        out[i * (k + 1) + k] = XR[i]
        out_names.append(names[i])
    return out, out_names, k + 1


def multi_interaction_columns(XR: np.ndarray, names: List[str], r: int, inter: np.ndarray):
    """One analysis per interaction column (-w; src/AIOwrapper.cpp:441-452, 1208-1241,
    names :618-660).  The reference reads file blocks of fmb = max(1, mb // k) SNPs
    (mb = min(m, 500)) and hands the solver, per block, k groups of that block's SNPs:
    group h holds, per SNP x, the r = 2 columns [I_h x, x], named "I<h>_<name>" and
    "I<h>_o_<name>".  Returns the columns in that order, their names, r = 2 and the
    solver's SNP block size fmb * k (its output blocks)."""
    if r != 1:
        raise ValueError("interactions need one column per SNP")
    k, m = inter.shape[0], XR.shape[0]
    fmb = max(1, min(m, 500) // k)
    out = np.empty((m * k * 2, XR.shape[1]), dtype=np.float32)
    out_names = []
    v = 0
    for b0 in range(0, m, fmb):
        for h in range(k):
            for i in range(b0, min(m, b0 + fmb)):
                out[2 * v] = inter[h] * XR[i]
                out[2 * v + 1] = XR[i]
                out_names += [f"I{h + 1}_{names[i]}", f"I{h + 1}_o_{names[i]}"]
                v += 1
    return out, out_names, 2, fmb * k


def erf_inv(z: float) -> float:
    """Inverse error function by Newton's method on math.erf (double precision)."""
    if z <= -1.0:
        return -math.inf
    if z >= 1.0:
        return math.inf
    if z == 0.0:
        return 0.0
    a = 0.147
    ln = math.log(1.0 - z * z)
    t1 = 2.0 / (math.pi * a) + ln / 2.0
    x = math.copysign(math.sqrt(math.sqrt(t1 * t1 - ln / a) - t1), z)
    c = 2.0 / math.sqrt(math.pi)
    for _ in range(100):
        step = (math.erf(x) - z) / (c * math.exp(-x * x))
        x -= step
        if abs(step) <= 1e-16 * (1.0 + abs(x)):
            break
    return x


def thresholds(s: Settings):
    """Effective store thresholds (src/Algorithm.cpp:338-342, 359; src/Utility.cpp:244-250).

    Returns (minR2store, minPstore, minTstore) as float32 values, the types
    the reference holds them in.
    """
    f32 = np.float32
    minR2store = f32(s.minR2store)
    minPstore = f32(s.minPstore)
    if f32(s.minR2disp) < minR2store or s.storeBin:
        minR2store = f32(s.minR2disp)
    if f32(s.minPdisp) > minPstore or s.storeBin:
        minPstore = f32(s.minPdisp)
    minT = f32(erf_inv(1.0 - float(minPstore)) * math.sqrt(2.0))
    return minR2store, minPstore, minT


def pvalue(t: float) -> float:
    """P of a |t| (src/Algorithm.cpp:1159-1167), double instead of long double."""
    if t < 1.6:
        t1 = float(np.float32(4.4 - t))
        return 0.5 - 0.1 * t1 * t
    return math.erfc(t * ONE_OVER_SQRT2)


# ----------------------------------------------------------------------------
# reader semantics
# ----------------------------------------------------------------------------
_HDR = struct.Struct("<H2xIIIIII5I")


def read_fvi(prefix: str):
    """Header fields and names of a .fvi file (src/AIOwrapper.cpp:2294-2317)."""
    raw = open(prefix + ".fvi", "rb").read()
    v = _HDR.unpack_from(raw, 0)
    nobs, nvar, nl = v[2], v[3], v[6]
    body = raw[48:]

    def name(i):
        b = body[i * nl:(i + 1) * nl]
        k = b.find(b"\0")
        return (b if k < 0 else b[:k]).decode("latin-1")

    return dict(n=nobs, v=nvar, namelength=nl,
                obs=[name(i) for i in range(nobs)],
                var=[name(nobs + i) for i in range(nvar)])


def read_fvd(prefix: str, n: int, v: int) -> np.ndarray:
    return np.fromfile(prefix + ".fvd", dtype="<f4", count=n * v).reshape(v, n)


def exclusion_rows(fname: str, n: int) -> np.ndarray:
    """0-based rows named by an exclusion list (src/AIOwrapper.cpp:2146-2233).

    Each line is ``first [second]`` (1-based, inclusive); a line with one
    number leaves ``second`` at its previous value and is read as a single
    index.  Reading stops once a range has reached ``n``.  Invalid files
    raise ValueError where the reference exits with status 1.
    """
    rows = []
    first = 0
    second = 0
    prev_second = -1
    with open(fname) as f:
        lines = f.read().splitlines()
    for line in lines:
        if second >= n:
            break
        tok = line.split()
        if len(tok) >= 1:          # a failed extraction leaves the variable unchanged
            first = int(tok[0])
        if len(tok) >= 2:
            second = int(tok[1])
        if prev_second > first:
            raise ValueError("exclusion list: indices not ordered")
        if second == prev_second:
            second = first
        else:
            if first > second:
                raise ValueError("exclusion list: pair not ordered")
            if first < 1 or second < 1:
                raise ValueError("exclusion list: non-positive index")
        prev_second = second
        rows.extend(range(first - 1, second))
    rows = np.unique(np.asarray([x for x in rows if 0 <= x < n], dtype=np.int64))
    if rows.size >= n:
        raise ValueError("exclusion list excluded all data")
    return rows


@dataclass
class Inputs:
    XL: np.ndarray      # (l, n) float32, kept rows
    XR: np.ndarray      # (m*r, n) float32, kept rows (NaN kept; imputed in solve)
    Y: np.ndarray       # (t, n) float32, kept rows (NaN kept)
    xl_names: List[str]
    xr_names: List[str]
    y_names: List[str]
    realN: int
    kept: np.ndarray
    r: int = 0          # columns per SNP of XR after a dosage model (0: Settings.r)
    mb: int = 0         # SNPs per output block (0: min(m, 500))


def load(xl_prefix: str, xr_prefix: str, y_prefix: str, s: Settings) -> Inputs:
    """Read the three inputs and apply the reference's row selection.

    Rows named in the exclusion list and rows with a NaN covariate are
    dropped (src/AIOwrapper.cpp:229-253, 1947-1991); realN is the row count
    before exclusions (src/AIOwrapper.cpp:87-90).
    """
    fl, fr, fy = read_fvi(xl_prefix), read_fvi(xr_prefix), read_fvi(y_prefix)
    n = fl["n"]
    if fr["v"] % s.r != 0:
        raise ValueError("numVariables of the genotype file is not a multiple of r")
    XL = read_fvd(xl_prefix, fl["n"], fl["v"])
    XR = read_fvd(xr_prefix, fr["n"], fr["v"])
    Y = read_fvd(y_prefix, fy["n"], fy["v"])
    keep = np.ones(n, dtype=bool)
    if s.fname_excludelist:
        keep[exclusion_rows(s.fname_excludelist, n)] = False
    keep &= ~np.isnan(XL).any(axis=0)
    inter = None
    if s.fname_interactions:
        # rows with a NaN interaction value leave the analysis (src/AIOwrapper.cpp:519-533)
        fi = read_fvi(s.fname_interactions)
        inter = read_fvd(s.fname_interactions, fi["n"], fi["v"])
        keep &= ~np.isnan(inter).any(axis=0)
    kept = np.nonzero(keep)[0]
    xr_names, r_eff = fr["var"], 0
    if s.model:
        XR, xr_names, r_eff = column_model(XR, xr_names, s)
    mb = 0
    if inter is not None and s.multi_interactions:
        XR, xr_names, r_eff, mb = multi_interaction_columns(XR, xr_names, r_eff or s.r, inter)
    elif inter is not None:
        XR, xr_names, r_eff = interaction_columns(XR, xr_names, r_eff or s.r, inter)
    return Inputs(XL=XL[:, kept], XR=XR[:, kept], Y=Y[:, kept],
                  xl_names=fl["var"], xr_names=xr_names, y_names=fy["var"],
                  realN=n, kept=kept, r=r_eff, mb=mb)


# ----------------------------------------------------------------------------
# the engine
# ----------------------------------------------------------------------------
@dataclass
class Dense:
    """Unfiltered per-test values: arrays indexed [trait, snp(, h)]."""
    beta: np.ndarray     # (t, m, p)
    se: np.ndarray       # (t, m, p)
    tstat: np.ndarray    # (t, m, p)
    rss: np.ndarray      # (t, m)
    r2: np.ndarray       # (t, m)
    nused: np.ndarray    # (t,)
    singular: np.ndarray  # (t, m) bool


@dataclass
class Results:
    """Stored results in reference output order, one entry per coefficient."""
    trait: np.ndarray
    snp: np.ndarray
    h: np.ndarray
    B: np.ndarray
    SE: np.ndarray
    T: np.ndarray
    P: np.ndarray
    R2: np.ndarray
    nUsed: np.ndarray
    nUsedPct: np.ndarray
    total_sig: int
    l: int
    r: int
    dense: Optional[Dense] = None
    meta: dict = field(default_factory=dict)


def _pair_products(XRc: np.ndarray, r: int):
    """Per SNP, the r x r products x_a*x_b over rows, as (m, r, r, n) views."""
    m = XRc.shape[0] // r
    X = XRc.reshape(m, r, -1)
    return X[:, :, None, :] * X[:, None, :, :]


def _masked_cross(M: np.ndarray, A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """out[t, a, b] = sum_k M[t, k] A[a, k] B[b, k]: per-trait sums over masked rows
    (the Stl_corr downdates, src/Algorithm.cpp:1324-1362), as one matrix product."""
    P = (A[:, None, :] * B[None, :, :]).reshape(-1, A.shape[1])
    return (M @ P.T).reshape(M.shape[0], A.shape[0], B.shape[0])


def _masked_snp_cross(M: np.ndarray, XL: np.ndarray, Xs: np.ndarray) -> np.ndarray:
    """out[t, i, a, b] = sum_k M[t, k] XL[a, k] Xs[i, b, k] (the Str_corr downdates,
    src/Algorithm.cpp:1260-1315), as one matrix product."""
    mc, r, n = Xs.shape
    l = XL.shape[0]
    P = (XL[None, :, None, :] * Xs[:, None, :, :]).reshape(mc * l * r, n)
    return (M @ P.T).reshape(M.shape[0], mc, l, r)


def _masked_snp_gram(M: np.ndarray, Xs: np.ndarray) -> np.ndarray:
    """out[t, i, a, b] = sum_k M[t, k] Xs[i, a, k] Xs[i, b, k] (the Sbr_corr downdates)."""
    mc, r, n = Xs.shape
    P = (Xs[:, :, None, :] * Xs[:, None, :, :]).reshape(mc * r * r, n)
    return (M @ P.T).reshape(M.shape[0], mc, r, r)


def solve(inp: Inputs, s: Settings, snp_chunk: int = 2048, keep_dense: bool = False) -> Results:
    r = inp.r or s.r
    XL = inp.XL.astype(np.float64)
    l, n = XL.shape
    p = l + r
    m = inp.XR.shape[0] // r
    t = inp.Y.shape[0]
    if p >= n:
        raise ValueError("p >= n")  # src/AIOwrapper.cpp:737-745
    minR2store, minPstore, minTstore = thresholds(s)
    minPdisp = float(np.float32(s.minPdisp))
    start_h = 1 if s.disp_cov else l

    # covariate rank check (src/Algorithm.cpp:497-522): any singular value < 1e-6
    sv = np.linalg.svd(XL.T, compute_uv=False)
    if np.any(sv < 1e-6):
        raise ValueError("covariate matrix has linearly dependent columns")

    # Y: NaN -> 0, missing sets and SST (src/Utility.cpp:329-378, src/Algorithm.cpp:1222-1251)
    Yraw = inp.Y.astype(np.float64)
    Mmask = np.isnan(Yraw)                        # (t, n) missing
    Y = np.where(Mmask, 0.0, Yraw)
    miss = Mmask.sum(axis=1)
    nobs = n - miss
    sx = Y.sum(axis=1)
    sxx = (Y * Y).sum(axis=1)
    SST = (sxx - sx * sx / nobs).astype(np.float32).astype(np.float64)
    Zmask = (Y == 0.0)                            # rows the RSS loop skips (includes missing)
    extra_zero = (Zmask & ~Mmask).any(axis=1)     # traits with observed exact zeros
    yy = (Y * Y).sum(axis=1)

    Stl = XL @ XL.T
    XLY = XL @ Y.T                                 # (l, t)
    Stl_corr = _masked_cross(Mmask.astype(np.float64), XL, XL)   # (t, l, l)
    Stl_zc = _masked_cross(Zmask.astype(np.float64), XL, XL)

    rec_trait, rec_snp, rec_h = [], [], []
    rec_B, rec_SE, rec_T, rec_R2 = [], [], [], []
    dense = None
    if keep_dense:
        dense = Dense(beta=np.zeros((t, m, p)), se=np.zeros((t, m, p)), tstat=np.zeros((t, m, p)),
                      rss=np.zeros((t, m)), r2=np.zeros((t, m)), nused=nobs.copy(),
                      singular=np.zeros((t, m), dtype=bool))

    for c0 in range(0, m, snp_chunk):
        c1 = min(m, c0 + snp_chunk)
        mc = c1 - c0
        XRc = inp.XR[c0 * r:c1 * r].astype(np.float64)
        # XR NaN -> column mean of the non-NaN entries (src/Utility.cpp:302-326)
        nanm = np.isnan(XRc)
        if nanm.any():
            cnt = n - nanm.sum(axis=1)
            avg = np.where(nanm, 0.0, XRc).sum(axis=1) / cnt
            XRc = np.where(nanm, avg[:, None], XRc)
        Xs = XRc.reshape(mc, r, n)

        # full (uncorrected) S per SNP (src/Algorithm.cpp:490-491, 633-661)
        Str = np.einsum("ak,ibk->iab", XL, Xs)                     # (mc, l, r)
        Sbr = np.einsum("iak,ibk->iab", Xs, Xs)                    # (mc, r, r)
        S = np.zeros((mc, p, p))
        S[:, :l, :l] = Stl
        S[:, :l, l:] = Str
        S[:, l:, :l] = np.transpose(Str, (0, 2, 1))
        S[:, l:, l:] = Sbr
        # var_x = diag(S^-1) of the uncorrected S (src/Algorithm.cpp:665-670)
        evs = np.linalg.eigvalsh(S)
        sing_full = evs[:, 0] <= 1e-12 * np.maximum(evs[:, -1], 1e-300)
        Sinv = np.linalg.inv(np.where(sing_full[:, None, None], np.eye(p), S))
        var_x = np.einsum("ihh->ih", Sinv)                          # (mc, p)

        # downdates per trait (src/Algorithm.cpp:1260-1362)
        Mf = Mmask.astype(np.float64)
        Str_c = _masked_snp_cross(Mf, XL, Xs)                       # (t, mc, l, r)
        Sbr_c = _masked_snp_gram(Mf, Xs)                            # (t, mc, r, r)
        Sj = np.broadcast_to(S, (t, mc, p, p)).copy()
        Sj[:, :, :l, :l] -= Stl_corr[:, None]
        if s.quirk_r2 and r >= 2:
            # correct_missings_S (src/Algorithm.cpp:1370-1399) on the upper
            # triangle that sposv('U') reads ([row, col] indexing here):
            #  * every SNP column's Str downdate is subtracted from column l only;
            #  * Sbr_corr[i*r+j] (row l+j, col l+i) is filled only for j < min(l, r) (:1300).
            Sbq = Sbr_c.copy()
            Sbq[:, :, min(l, r):, :] = 0.0
            Sj[:, :, l:, l:] -= Sbq
            Sj[:, :, :l, l] -= Str_c.sum(axis=3)
            U = np.triu(Sj)
            Sj = U + np.transpose(U, (0, 1, 3, 2)) - U * np.eye(p)
        else:
            Sj[:, :, :l, l:] -= Str_c
            Sj[:, :, l:, :l] -= np.transpose(Str_c, (0, 1, 3, 2))
            Sj[:, :, l:, l:] -= Sbr_c

        # right-hand sides [XL'y; XR_i'y] (src/Algorithm.cpp:583-585, 705-707, 734-736)
        XRY = (Y @ Xs.reshape(mc * r, n).T).reshape(t, mc, r)       # (t, mc, r)
        rhs = np.concatenate([np.broadcast_to(XLY.T[:, None, :], (t, mc, l)), XRY], axis=2)

        # b = S \ rhs (src/Algorithm.cpp:767-768)
        ev = np.linalg.eigvalsh(Sj)
        sing = (ev[..., 0] <= 1e-12 * np.maximum(ev[..., -1], 1e-300)) | sing_full[None, :]
        Ssafe = np.where(sing[..., None, None], np.eye(p), Sj)
        beta = np.linalg.solve(Ssafe, rhs[..., None])[..., 0]       # (t, mc, p)

        # RSS over rows with y != 0 (src/Algorithm.cpp:976-1024), exact expansion:
        # RSS = y'y - 2 b'X'y + b' G b with G the Gram matrix of those rows
        G = np.broadcast_to(S, (t, mc, p, p)).copy()
        Zf = Zmask.astype(np.float64)
        G[:, :, :l, :l] -= Stl_zc[:, None]
        Strz = _masked_snp_cross(Zf, XL, Xs)
        G[:, :, :l, l:] -= Strz
        G[:, :, l:, :l] -= np.transpose(Strz, (0, 1, 3, 2))
        G[:, :, l:, l:] -= _masked_snp_gram(Zf, Xs)
        rss = (yy[:, None] - 2.0 * (beta * rhs).sum(axis=2)
               + (beta[..., None, :] @ G @ beta[..., :, None])[..., 0, 0])

        # statistics (src/Algorithm.cpp:1034-1134)
        ncorr = (n - miss - p).astype(np.float64)                   # n_corrected
        varFactor = ((ncorr + p) / n)[:, None]
        R2 = 1.0 - (rss / (ncorr[:, None] - 1.0)) / (SST[:, None] / (n - 1.0))
        sig = np.sqrt(np.maximum(rss, 0.0) / ncorr[:, None])
        with np.errstate(invalid="ignore", divide="ignore"):
            SE = sig[..., None] * np.sqrt(var_x[None] * varFactor[..., None])
            T = np.abs(beta / SE)

        if keep_dense:
            dense.beta[:, c0:c1] = beta
            dense.se[:, c0:c1] = SE
            dense.tstat[:, c0:c1] = T
            dense.rss[:, c0:c1] = rss
            dense.r2[:, c0:c1] = R2
            dense.singular[:, c0:c1] = sing

        # filters (src/Algorithm.cpp:1119-1203)
        r2ok = (R2 > float(minR2store)) | s.storePInd
        live = (rss > 0.0) & r2ok & ~sing
        for hh in range(p - 1, start_h - 1, -1):
            stored = live & ((T[..., hh] > float(minTstore)) | s.storePInd)
            tj, ti = np.nonzero(stored)
            rec_trait.append(tj)
            rec_snp.append(ti + c0)
            rec_h.append(np.full(tj.size, hh))
            rec_B.append(beta[tj, ti, hh])
            rec_SE.append(SE[tj, ti, hh])
            rec_T.append(T[tj, ti, hh])
            rec_R2.append(R2[tj, ti])

    trait = np.concatenate(rec_trait) if rec_trait else np.zeros(0, int)
    snp = np.concatenate(rec_snp) if rec_snp else np.zeros(0, int)
    h = np.concatenate(rec_h) if rec_h else np.zeros(0, int)
    B = np.concatenate(rec_B) if rec_B else np.zeros(0)
    SEa = np.concatenate(rec_SE) if rec_SE else np.zeros(0)
    Ta = np.concatenate(rec_T) if rec_T else np.zeros(0)
    R2a = np.concatenate(rec_R2) if rec_R2 else np.zeros(0)

    # every stored result with P < minPdisp counts, whether or not its row is
    # kept below (src/Algorithm.cpp:1189-1192)
    P_all = np.array([pvalue(float(np.float32(x))) for x in Ta])
    total_sig = int(np.sum(minPdisp > P_all))

    # a row survives only if one of its SNP terms was stored (src/Algorithm.cpp:1156-1157, 1197)
    key_row = trait.astype(np.int64) * m + snp
    has_snp_term = np.zeros(t * m, dtype=bool)
    has_snp_term[key_row[h >= l]] = True
    keep = has_snp_term[key_row]
    trait, snp, h, B, SEa, Ta, R2a = (a[keep] for a in (trait, snp, h, B, SEa, Ta, R2a))

    # reference order: Y block, SNP block, trait, SNP, h descending
    tb, mb = min(t, 1000), (inp.mb or min(m, 500))
    order = np.lexsort((-h, snp, trait, snp // mb, trait // tb))
    trait, snp, h, B, SEa, Ta, R2a = (a[order] for a in (trait, snp, h, B, SEa, Ta, R2a))
    P = np.array([pvalue(float(np.float32(x))) for x in Ta])
    nUsed = (n - miss)[trait]
    nUsedPct = (nUsed.astype(np.float32) / np.float32(inp.realN)).astype(np.float32)
    return Results(trait=trait, snp=snp, h=h, B=B, SE=SEa, T=Ta, P=P, R2=R2a,
                   nUsed=nUsed, nUsedPct=nUsedPct, total_sig=total_sig, l=l, r=r,
                   dense=dense, meta=dict(minTstore=float(minTstore), minR2store=float(minR2store),
                                          minPdisp=minPdisp, extra_zero_traits=int(extra_zero.sum())))


def displayed(res: Results, s: Settings) -> np.ndarray:
    """Mask of stored results that go to _dis.txt (src/AIOwrapper.cpp:1494)."""
    if s.storePInd:
        return np.ones(res.T.size, dtype=bool)
    return (res.P <= float(np.float32(s.minPdisp))) & (res.R2.astype(np.float32) >= np.float32(s.minR2disp))


def run_files(xl: str, xr: str, y: str, s: Settings, **kw) -> tuple[Results, Inputs]:
    inp = load(xl, xr, y, s)
    return solve(inp, s, **kw), inp


def result_names(res: Results, inp: Inputs, l: int, r: int):
    """(trait name, SNP-column text) of each stored result, as _dis.txt spells them.

    SNP terms print as " <ARname>", covariate terms as "<ALname>:<ARname>"
    where ARname is the SNP's first column (src/AIOwrapper.cpp:1497-1505).
    """
    out = []
    for tr, sn, hh in zip(res.trait, res.snp, res.h):
        if hh >= l:
            a = " " + inp.xr_names[sn * r + (hh - l)]
        else:
            a = inp.xl_names[hh] + ":" + inp.xr_names[sn * r]
        out.append((inp.y_names[tr], a))
    return out


def parse_dis(path: str):
    """Parse a _dis.txt file into a list of dicts (numeric fields as float)."""
    rows = []
    with open(path) as f:
        head = f.readline().rstrip("\n").split("\t")
        if head != ["Phe", "SNP", "n", "nPct", "B", "R2", "SE", "T", "P"]:
            raise ValueError(f"{path}: unexpected header {head}")
        for line in f:
            c = line.rstrip("\n").split("\t")
            rows.append(dict(Phe=c[0], SNP=c[1], n=int(c[2]), nPct=c[3], B=float(c[4]),
                             R2=float(c[5]), SE=float(c[6]), T=float(c[7]), P=c[8]))
    return rows


if __name__ == "__main__":  # pragma: no cover - manual use
    import sys
    pre = sys.argv[1]
    res, inp = run_files(pre + "XL", pre + "XR", pre + "Y", Settings(storePInd="-f" in sys.argv))
    print(len(res.T), res.total_sig, os.path.basename(pre))
