"""Seeded synthetic association-scan inputs with the shapes of the benchmark workloads.

No public dataset is involved: every workload is drawn from numpy's PCG64
with a fixed seed.  The distributions follow the workload descriptions:

* covariates XL = [intercept, sex ~ Bernoulli(0.5), age ~ N(50, 10), PCs ~ N(0,1)...]
  (optionally a near-collinear ``age2 = age + N(0, 1e-3)`` column);
* dosages  x = clip(Binomial(2, maf) + U(-0.05, 0.05), 0, 2) rounded to 0.001,
  ``maf ~ U(maf_lo, maf_hi)`` (a fraction of SNPs may be drawn from a low-MAF band);
* r = 2 SNPs carry the SNP x sex interaction column first, then the SNP
  itself ([INT*X, X], the column order of the reference's interaction
  generator, src/AIOwrapper.cpp:808-840);
* traits y_j = XL b_j + effect * x_causal(j) + N(0, s_j^2),  b_j ~ N(0, 1),
  ``s_j^2 ~ U(noise_lo, noise_hi)``, causal SNP of trait j is SNP ``j mod m``;
* missing phenotypes (NaN) either uniformly per trait or drawn from a fixed
  number of missingness patterns (traits sharing a pattern share the NaN rows).

Arrays are variable-major ``(v, n)`` float32, the layout of ``.fvd`` files.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import fvformat


@dataclass
class Workload:
    n: int
    m: int
    t: int
    l: int = 3
    r: int = 1
    maf_lo: float = 0.05
    maf_hi: float = 0.5
    low_maf_frac: float = 0.0          # fraction of SNPs with maf in [0.005, 0.01]
    collinear: bool = False            # append age2 = age + N(0, 1e-3)
    noise_lo: float = 1.0
    noise_hi: float = 1.0
    effect: float = 0.1
    miss_mode: str = "uniform"         # "uniform" | "patterns" | "none"
    miss_frac: float = 0.05            # uniform mode: fraction of NaNs per trait
    n_patterns: int = 0                # patterns mode: number of distinct patterns
    miss_hi: float = 0.10              # patterns mode: per-pattern fraction ~ U(0, miss_hi)
    zipf: float = 0.0                  # patterns mode: Zipf exponent of group sizes (0: uniform)
    group_max: int = 0                 # patterns mode: largest group size with Zipf sizes
    xr_nan_frac: float = 0.0           # fraction of NaN dosages (mean-imputed by the engine)
    xl_nan_rows: int = 0               # rows with a NaN covariate (dropped by the reader)
    prob_cols: int = 0                 # 2 or 3: genotype-probability columns per SNP (AA, AB[, BB])
                                       # instead of one dosage column (input of the dosage models)
    seed: int = 0
    name: str = "custom"


# The five benchmark workloads (sizes as specified; tests scale them down).
CONFIGS = {
    0: Workload(n=1000, m=10000, t=100, l=3, r=1, maf_lo=0.05, maf_hi=0.5,
                miss_mode="uniform", miss_frac=0.05, seed=1000, name="plain-fp32-cpu"),
    1: Workload(n=10000, m=500000, t=1000, l=4, r=1, maf_lo=0.01, maf_hi=0.5,
                noise_lo=0.5, noise_hi=2.0, miss_mode="patterns", n_patterns=20,
                miss_hi=0.10, seed=1001, name="plain-fp32-omics"),
    2: Workload(n=10000, m=500000, t=1000, l=5, r=1, maf_lo=0.01, maf_hi=0.5,
                low_maf_frac=0.01, collinear=True, noise_lo=0.5, noise_hi=2.0,
                miss_mode="patterns", n_patterns=20, miss_hi=0.10, seed=1002,
                name="mixed-collinear"),
    3: Workload(n=8000, m=200000, t=2000, l=5, r=2, maf_lo=0.05, maf_hi=0.5,
                miss_mode="patterns", n_patterns=150, miss_hi=0.15, zipf=1.2,
                group_max=400, seed=1003, name="batched-interaction"),
}


def scaled(cfg: int | Workload, **over) -> Workload:
    """A copy of a workload with some fields replaced (e.g. smaller n/m/t)."""
    base = CONFIGS[cfg] if isinstance(cfg, int) else cfg
    d = dict(base.__dict__)
    d.update(over)
    return Workload(**d)


def _zipf_sizes(rng, groups: int, total: int, s: float, cap: int) -> np.ndarray:
    """Group sizes proportional to rank^-s, each in [1, cap], summing to ``total``."""
    w = np.arange(1, groups + 1, dtype=np.float64) ** (-s)
    sizes = np.maximum(1, np.floor(w / w.sum() * total)).astype(np.int64)
    sizes = np.minimum(sizes, cap)
    # distribute the remainder over groups that still have room, largest first
    rest = total - int(sizes.sum())
    i = 0
    while rest != 0:
        g = i % groups
        if rest > 0 and sizes[g] < cap:
            sizes[g] += 1
            rest -= 1
        elif rest < 0 and sizes[g] > 1:
            sizes[g] -= 1
            rest += 1
        i += 1
        if i > 100 * groups * max(1, abs(rest)):
            raise ValueError("cannot fit group sizes")
    rng.shuffle(sizes)
    return sizes


@dataclass
class Dataset:
    XL: np.ndarray          # (l, n) float32
    XR: np.ndarray          # (m*r, n) float32
    Y: np.ndarray           # (t, n) float32 with NaN for missing
    xl_names: List[str]
    xr_names: List[str]
    y_names: List[str]
    obs: List[str]
    pattern_of_trait: Optional[np.ndarray] = None
    causal: Optional[np.ndarray] = None
    meta: dict = field(default_factory=dict)


def covariates(rng, w: Workload) -> tuple[np.ndarray, List[str]]:
    n = w.n
    cols = [np.ones(n), rng.binomial(1, 0.5, n).astype(np.float64), rng.normal(50.0, 10.0, n)]
    names = ["intercept", "sex", "age"]
    npc = w.l - 3 - (1 if w.collinear else 0)
    for i in range(max(0, npc)):
        cols.append(rng.normal(0.0, 1.0, n))
        names.append(f"pc{i + 1}")
    if w.collinear:
        cols.append(cols[2] + rng.normal(0.0, 1e-3, n))
        names.append("age2")
    XL = np.stack(cols[: w.l]).astype(np.float32)
    return XL, names[: w.l]


def dosages(rng, n: int, m: int, maf_lo: float, maf_hi: float,
            low_maf_frac: float = 0.0) -> np.ndarray:
    maf = rng.uniform(maf_lo, maf_hi, m)
    if low_maf_frac > 0:
        k = int(round(low_maf_frac * m))
        idx = rng.choice(m, k, replace=False)
        maf[idx] = rng.uniform(0.005, 0.01, k)
    g = rng.binomial(2, maf[:, None], (m, n)).astype(np.float64)
    g += rng.uniform(-0.05, 0.05, (m, n))
    return np.round(np.clip(g, 0.0, 2.0), 3).astype(np.float32)


def genotype_probabilities(rng, n: int, m: int, maf_lo: float, maf_hi: float, cols: int):
    """Imputed genotype probabilities: genotype g ~ Binomial(2, maf) (copies of
    the counted allele), its class AA (g = 2), AB (g = 1) or BB (g = 0) gets
    1 - e with e ~ U(0, 0.3), the other two classes share e; rounded to 0.001.
    Returns the (m*cols, n) file columns [P(AA), P(AB)(, P(BB))] per SNP, the
    additive dosage 2 P(AA) + P(AB) (m, n) and the column names."""
    if cols not in (2, 3):
        raise ValueError("genotype probabilities come as 2 or 3 columns per SNP")
    maf = rng.uniform(maf_lo, maf_hi, m)
    g = rng.binomial(2, maf[:, None], (m, n))
    e = rng.uniform(0.0, 0.3, (m, n))
    split = rng.uniform(0.0, 1.0, (m, n))
    P = np.empty((m, 3, n))
    for cls, gval in enumerate((2, 1, 0)):
        hit = g == gval
        others = [c for c in range(3) if c != cls]
        P[:, cls][hit] = 1.0 - e[hit]
        P[:, others[0]][hit] = e[hit] * split[hit]
        P[:, others[1]][hit] = e[hit] * (1.0 - split[hit])
    P = np.round(P, 3).astype(np.float32)
    XR = np.ascontiguousarray(P[:, :cols].reshape(m * cols, n))
    X = (2.0 * P[:, 0] + P[:, 1]).astype(np.float32)
    names = []
    for i in range(m):
        names += [f"snp{i + 1}_{c}" for c in ("AA", "AB", "BB")[:cols]]
    return XR, X, names


def generate(w: Workload) -> Dataset:
    """Draw one workload in memory.  Meant for n*m up to a few 1e8."""
    rng = np.random.Generator(np.random.PCG64(w.seed))
    n, m, t, r = w.n, w.m, w.t, w.r
    XL, xl_names = covariates(rng, w)
    if w.prob_cols:
        XR, X, xr_names = genotype_probabilities(rng, n, m, w.maf_lo, w.maf_hi, w.prob_cols)
    else:
        X = dosages(rng, n, m, w.maf_lo, w.maf_hi, w.low_maf_frac)
    if w.prob_cols:
        pass
    elif r == 1:
        XR = X
        xr_names = [f"snp{i + 1}" for i in range(m)]
    elif r == 2:
        sex = XL[1]
        XR = np.empty((2 * m, n), dtype=np.float32)
        XR[0::2] = X * sex[None, :]
        XR[1::2] = X
        xr_names = []
        for i in range(m):
            xr_names += [f"snp{i + 1}_sx", f"snp{i + 1}"]
    else:
        raise ValueError("synthetic workloads use r = 1 or r = 2")
    if w.xr_nan_frac > 0:
        mask = rng.random(XR.shape) < w.xr_nan_frac
        XR = XR.copy()
        XR[mask] = np.nan

    causal = np.arange(t) % m
    b = rng.normal(0.0, 1.0, (t, XL.shape[0]))
    noise_sd = np.sqrt(rng.uniform(w.noise_lo, w.noise_hi, t))
    Y = b @ XL.astype(np.float64) + w.effect * X[causal].astype(np.float64)
    Y += rng.normal(0.0, 1.0, (t, n)) * noise_sd[:, None]

    pattern_of_trait = None
    if w.miss_mode == "uniform":
        k = int(round(w.miss_frac * n))
        for j in range(t):
            Y[j, rng.choice(n, k, replace=False)] = np.nan
    elif w.miss_mode == "patterns":
        G = w.n_patterns
        if w.zipf > 0:
            sizes = _zipf_sizes(rng, G, t, w.zipf, w.group_max or t)
            pattern_of_trait = np.repeat(np.arange(G), sizes)
            rng.shuffle(pattern_of_trait)
        else:
            pattern_of_trait = rng.integers(0, G, t)
        frac = rng.uniform(0.0, w.miss_hi, G)
        for g in range(G):
            rows = rng.choice(n, int(round(frac[g] * n)), replace=False)
            sel = np.nonzero(pattern_of_trait == g)[0]
            if rows.size and sel.size:
                Y[np.ix_(sel, rows)] = np.nan
    elif w.miss_mode != "none":
        raise ValueError(w.miss_mode)

    if w.xl_nan_rows > 0:
        XL = XL.copy()
        rows = rng.choice(n, w.xl_nan_rows, replace=False)
        cols = rng.integers(1, XL.shape[0], w.xl_nan_rows)
        XL[cols, rows] = np.nan

    Y = Y.astype(np.float32)
    return Dataset(XL=XL, XR=XR, Y=Y, xl_names=xl_names, xr_names=xr_names,
                   y_names=[f"ph{j + 1}" for j in range(t)], obs=fvformat.obs_names(n),
                   pattern_of_trait=pattern_of_trait, causal=causal,
                   meta={"workload": w.name, "seed": w.seed})


def write_dataset(ds: Dataset, prefix: str) -> dict:
    """Write XL/XR/Y as ``{prefix}XL.fv*``, ``{prefix}XR.fv*``, ``{prefix}Y.fv*``."""
    paths = {"XL": prefix + "XL", "XR": prefix + "XR", "Y": prefix + "Y"}
    fvformat.write_fv(paths["XL"], ds.XL, ds.obs, ds.xl_names)
    fvformat.write_fv(paths["XR"], ds.XR, ds.obs, ds.xr_names)
    fvformat.write_fv(paths["Y"], ds.Y, ds.obs, ds.y_names)
    return paths


def generate_device(w: Workload, device, seed_offset: int = 0, snp_chunk: int = 32768):
    """Draw a workload directly in device memory with torch (for full-size runs).

    Same distributions as ``generate`` (different random stream).  Returns
    (XL (l, n), XR (m*r, n), Y (t, n)) float32 CUDA tensors, plus the pattern
    of each trait.  Used by the benchmark, where numpy on the host would take
    minutes for the 20 GB genotype matrix.
    """
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(w.seed * 1000003 + seed_offset)
    n, m, t, r = w.n, w.m, w.t, w.r
    f32 = torch.float32
    cols = [torch.ones(n, device=device), (torch.rand(n, generator=g, device=device) < 0.5).to(f32),
            50.0 + 10.0 * torch.randn(n, generator=g, device=device)]
    npc = w.l - 3 - (1 if w.collinear else 0)
    for _ in range(max(0, npc)):
        cols.append(torch.randn(n, generator=g, device=device))
    if w.collinear:
        cols.append(cols[2] + 1e-3 * torch.randn(n, generator=g, device=device))
    XL = torch.stack(cols[: w.l]).contiguous()
    maf = w.maf_lo + (w.maf_hi - w.maf_lo) * torch.rand(m, generator=g, device=device)
    if w.low_maf_frac > 0:
        k = int(round(w.low_maf_frac * m))
        idx = torch.randperm(m, generator=g, device=device)[:k]
        maf[idx] = 0.005 + 0.005 * torch.rand(k, generator=g, device=device)
    XR = torch.empty((m * r, n), dtype=f32, device=device)
    for c0 in range(0, m, snp_chunk):
        c1 = min(m, c0 + snp_chunk)
        p = maf[c0:c1, None]
        x = (torch.rand((c1 - c0, n), generator=g, device=device) < p).to(f32)
        x += (torch.rand((c1 - c0, n), generator=g, device=device) < p).to(f32)
        x += 0.1 * torch.rand((c1 - c0, n), generator=g, device=device) - 0.05
        x = torch.round(x.clamp_(0.0, 2.0) * 1000.0) / 1000.0
        if r == 1:
            XR[c0:c1] = x
        else:
            XR[2 * c0:2 * c1:2] = x * XL[1][None, :]
            XR[2 * c0 + 1:2 * c1:2] = x
        del x
    causal = torch.arange(t, device=device) % m
    b = torch.randn((t, w.l), generator=g, device=device)
    noise = torch.sqrt(w.noise_lo + (w.noise_hi - w.noise_lo) * torch.rand(t, generator=g, device=device))
    xc = XR[causal * r + (r - 1)]
    Y = b @ XL + w.effect * xc + torch.randn((t, n), generator=g, device=device) * noise[:, None]
    pattern = None
    if w.miss_mode == "patterns":
        G = w.n_patterns
        if w.zipf > 0:
            rng = np.random.Generator(np.random.PCG64(w.seed + seed_offset))
            sizes = _zipf_sizes(rng, G, t, w.zipf, w.group_max or t)
            pat = np.repeat(np.arange(G), sizes)
            rng.shuffle(pat)
            pattern = torch.as_tensor(pat, device=device)
        else:
            pattern = torch.randint(0, G, (t,), generator=g, device=device)
        frac = w.miss_hi * torch.rand(G, generator=g, device=device)
        miss = torch.rand((G, n), generator=g, device=device) < frac[:, None]
        Y = torch.where(miss[pattern], torch.full_like(Y, float("nan")), Y)
    elif w.miss_mode == "uniform":
        miss = torch.rand((t, n), generator=g, device=device) < w.miss_frac
        Y = torch.where(miss, torch.full_like(Y, float("nan")), Y)
    return XL, XR, Y.contiguous(), pattern
