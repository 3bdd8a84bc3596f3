"""Datasets of the quirk-mode dense tests (the reference's r >= 2 downdate,
src/Algorithm.cpp:1300, 1390-1396, reproduced by the engine and the oracle).

Shared by tests/test_gpu_parity.py and tests/golden/measure_quirk_noise.py,
which measures the reference's own deviation from the FP64 oracle on them.
"""
import numpy as np

from omicabelnomm_b200 import synth

CASES = ("r2_missing", "r2_yzero_l1", "r3_missing", "r5_l2")

R2_MISSING = dict(n=600, m=120, t=16, l=5, r=2, miss_mode="patterns", n_patterns=4, miss_hi=0.15, seed=26)


def multicol(r, seed, **over):
    """r dosage columns per SNP: consecutive independent dosage columns grouped r at a time."""
    w = dict(n=500, m=30, t=12, l=4, miss_mode="patterns", n_patterns=3, miss_hi=0.12)
    w.update(over)
    w["m"] *= r
    return synth.generate(synth.scaled(0, seed=seed, **w))


def yzero(ds, seed):
    """Six observed phenotype values per trait set to exactly 0 (zero sets)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    for j in range(ds.Y.shape[0]):
        obs = np.nonzero(~np.isnan(ds.Y[j]))[0]
        ds.Y[j, rng.choice(obs, 6, replace=False)] = 0.0
    return ds


def build(case):
    """(r, dataset) of one case: r = 2 with l = 5; r = 2 with one covariate and
    zero sets (r > l); r = 3; r = 5 with l = 2 (padding columns in the kernels)."""
    if case == "r2_missing":
        return 2, synth.generate(synth.scaled(0, **R2_MISSING))
    if case == "r2_yzero_l1":
        return 2, yzero(multicol(2, 74, n=500, m=45, l=1, n_patterns=3, miss_hi=0.15), 9)
    if case == "r3_missing":
        return 3, multicol(3, 75)
    if case == "r5_l2":
        return 5, multicol(5, 76, l=2)
    raise KeyError(case)
