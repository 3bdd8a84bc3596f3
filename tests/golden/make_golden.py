"""Generate the golden fixtures: outputs of the reference CLI on seeded inputs.

Run in a container where the reference tree is present and the reference
CLI has been compiled from its own sources (``make -C oracle``):

    python tests/golden/make_golden.py

For every case in CASES this script

1. draws the inputs with ``omicabelnomm_b200.synth`` (seeded, so the test
   suite regenerates them byte for byte; the manifest keeps their sha256),
2. runs ``oracle/_ref/omicabelnomm_ref`` with the case's flags (for the
   dosage models -j/-k/-l, which the reference's command line rejects,
   ``oracle/_ref/ref_model_driver``: its solver with the model set in-process),
3. stores the reference's ``_dis.txt`` (gzip) and, with ``-b``, its
   ``_sto.ibin`` / ``_sto.dbin`` plus the printed "Number of Significant
   Results" in ``tests/golden/<case>/``.

The inputs themselves are not committed; only these outputs are.
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from omicabelnomm_b200 import synth  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "omicabelnomm_ref")
# the reference's solver with a dosage model set in-process (its CLI cannot reach the models)
REF_MODEL = os.path.join(ROOT, "oracle", "_ref", "ref_model_driver")
MODEL_FLAGS = {"-j": 0, "-k": 1, "-l": 2, "-z": 3, "-y": 4}   # the reference's Settings::model values

# name -> (workload overrides on config 0, post-processing, [flag sets])
CASES = {
    # plain r = 1, 5 % uniform NaN per trait
    "r1_uniform": (dict(n=400, m=120, t=12, seed=11), None,
                   [["-f"], [], ["-i"], ["-f", "-i"], ["-b"], ["-b", "-i"], ["-b", "-f"]]),
    # shared missingness patterns, two SNP blocks (m > 500)
    "r1_patterns": (dict(n=300, m=620, t=6, l=4, miss_mode="patterns", n_patterns=3,
                         miss_hi=0.1, seed=12), None, [["-f"], [], ["-b"]]),
    # two trait blocks (t > 1000)
    "r1_tblocks": (dict(n=60, m=3, t=1010, seed=13), None, [[], ["-b"]]),
    # covariate NaNs and an exclusion list drop individuals
    "r1_exclude": (dict(n=300, m=80, t=8, xl_nan_rows=7, seed=14), "exclude",
                   [["-f", "-x", "{excl}"], ["-x", "{excl}", "-b"]]),
    # NaN dosages are mean-imputed
    "r1_xrnan": (dict(n=300, m=80, t=8, xr_nan_frac=0.02, seed=15), None, [["-f"]]),
    # observed phenotypes that are exactly 0 are skipped by the RSS loop
    "r1_yzero": (dict(n=300, m=80, t=8, seed=16), "yzero", [["-f"]]),
    # strong planted effects: trait j with SNP j (known-answer structure)
    "r1_strong": (dict(n=500, m=40, t=20, effect=1.0, seed=17), None, [[], ["-b"]]),
    # r = 2 (SNP x sex, SNP) without phenotype missingness
    "r2_complete": (dict(n=400, m=60, t=6, l=4, r=2, miss_mode="none", seed=18), None,
                    [["-n", "2", "-f"], ["-n", "2", "-i"], ["-n", "2", "-b"]]),
    # r = 2 with missingness (the reference's downdate bug applies)
    "r2_missing": (dict(n=400, m=60, t=6, l=4, r=2, seed=19), None, [["-n", "2", "-f"]]),
    # dosage models on genotype probabilities: three columns (AA, AB, BB) per SNP
    "r1_dos3": (dict(n=400, m=60, t=8, prob_cols=3, seed=31), None,
                [["-n", "3", "-j"], ["-n", "3", "-k"], ["-n", "3", "-l"], ["-n", "3", "-j", "-b"],
                 ["-n", "3", "-k", "-f"]]),
    # ... and two columns (AA, AB)
    "r1_dos2": (dict(n=300, m=50, t=6, prob_cols=2, seed=32), None,
                [["-n", "2", "-j"], ["-n", "2", "-k", "-b"]]),
    # custom models with a factors file on (AA, AB): linear (each column scaled, r = 2; with all
    # three columns, which sum to 1, the model would be collinear with the intercept) and additive
    "r1_dosf": (dict(n=400, m=40, t=6, prob_cols=2, seed=33), "factors",
                [["-n", "2", "-z", "{fac}"], ["-n", "2", "-y", "{fac}"], ["-n", "2", "-y", "{fac}", "-b"]]),
    # single-set interactions (-v): SNP x I and the SNP itself (r = 2); no phenotype missingness, so
    # the reference's r >= 2 downdate quirk does not enter; a few NaN interaction values drop rows
    "r1_inter": (dict(n=400, m=50, t=6, l=4, miss_mode="none", seed=34), "inter",
                 [["-v", "{inter}"], ["-v", "{inter}", "-b"], ["-v", "{inter}", "-f", "-i"]]),
    # three interaction columns (r = 4)
    "r1_inter3": (dict(n=400, m=30, t=5, l=3, miss_mode="none", seed=35), "inter3",
                  [["-v", "{inter}"], ["-v", "{inter}", "-f"]]),
    # one analysis per interaction column (-w, three columns): r = 2 ([I_h x, x]) per (SNP, column);
    # 230 SNPs make reference blocks of 76 file SNPs x 3 columns and a ragged last block of 2.
    # With -b only the .dbin is kept: the reference's .ibin name list reads past its name table
    # here (it writes fileR * m names with m already multiplied by the column count)
    "r1_multinter": (dict(n=300, m=230, t=5, l=3, miss_mode="none", seed=36), "inter3",
                     [["-w", "{inter}"], ["-w", "{inter}", "-f"], ["-w", "{inter}", "-f", "-i"],
                      ["-w", "{inter}", "-b"]]),
    # three columns per SNP without a model (-n 3: consecutive triples of dosage columns form one SNP);
    # the engine runs them as four columns with a zero column added on the device
    "r3_cols": (dict(n=400, m=120, t=5, l=4, miss_mode="none", seed=37), None,
                [["-n", "3"], ["-n", "3", "-f"], ["-n", "3", "-b"]]),
    # ... with phenotype missingness: the reference's r >= 2 downdate applies
    "r3_missing": (dict(n=400, m=90, t=6, l=4, seed=38), None, [["-n", "3", "-f"]]),
    # two interaction columns (-v, r = 3) and four (r = 5: eight kernel columns per SNP)
    "r1_inter2": (dict(n=400, m=40, t=5, l=3, miss_mode="none", seed=39), "inter2",
                  [["-v", "{inter}"], ["-v", "{inter}", "-f"]]),
    "r1_inter4": (dict(n=400, m=30, t=4, l=3, miss_mode="none", seed=40), "inter4",
                  [["-v", "{inter}"], ["-v", "{inter}", "-f"]]),
}

FACTORS = "0.5 1.5\n"


def interaction_file(n: int, seed: int, prefix: str, k: int):
    """k interaction columns of n individuals: N(0, 1), then Bernoulli(0.5), then U(0, 2), then
    N(1, 0.5); the first column holds 3 NaN values."""
    import numpy as np
    from omicabelnomm_b200 import fvformat
    rng = np.random.Generator(np.random.PCG64(seed))
    cols = [rng.normal(0.0, 1.0, n), rng.binomial(1, 0.5, n).astype(np.float64), rng.uniform(0.0, 2.0, n)]
    nan_rows = rng.choice(n, 3, replace=False)
    if k > 3:
        cols.append(rng.normal(1.0, 0.5, n))
    I = np.stack(cols[:k]).astype(np.float32)
    I[0, nan_rows] = np.nan
    fvformat.write_fv(prefix, I, fvformat.obs_names(n), ["inter_env", "inter_sex", "inter_dose", "inter_score"][:k])

EXCLUDE_LIST = "1 2\n5\n7\n9 11\n13\n40 44\n"


def build_inputs(case: str, where: str):
    over, post, _ = CASES[case]
    w = synth.scaled(0, **over)
    ds = synth.generate(w)
    if post == "yzero":
        # set a few observed entries of every trait to exactly zero
        import numpy as np
        rng = np.random.Generator(np.random.PCG64(w.seed + 99))
        for j in range(ds.Y.shape[0]):
            obs = np.nonzero(~np.isnan(ds.Y[j]))[0]
            ds.Y[j, rng.choice(obs, 5, replace=False)] = 0.0
    pre = os.path.join(where, case + "_")
    synth.write_dataset(ds, pre)
    extra = {}
    if post == "exclude":
        p = os.path.join(where, case + "_excl.txt")
        with open(p, "w") as f:
            f.write(EXCLUDE_LIST)
        extra["excl"] = p
    if post in ("inter", "inter2", "inter3", "inter4"):
        p = os.path.join(where, case + "_INT")
        interaction_file(over["n"], over["seed"] + 7, p, {"inter": 1, "inter2": 2, "inter3": 3, "inter4": 4}[post])
        extra["inter"] = p
    if post == "factors":
        p = os.path.join(where, case + "_factors.txt")
        with open(p, "w") as f:
            f.write(FACTORS)
        extra["fac"] = p
    return pre, extra


def sha256(path: str) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for blk in iter(lambda: f.read(1 << 20), b""):
            h.update(blk)
    return h.hexdigest()


def input_digests(pre: str) -> dict:
    return {k: sha256(pre + k + ".fvd") for k in ("XL", "XR", "Y")} | \
           {k + ".fvi": sha256(pre + k + ".fvi") for k in ("XL", "XR", "Y")}


def flag_tag(flags) -> str:
    t = "".join(f.strip("-") for f in flags if not f.startswith("{") and not f.isdigit()
                and f != "{excl}")
    return t or "default"


def ref_command(flags, pre: str, extra: dict, out: str, threads: int = 0):
    """Command line of the reference run with these flags (the CLI, or the in-process model
    driver for the dosage models and interactions); threads > 0 adds the thread count."""
    args = [f.format(**extra) for f in flags]
    model = [f for f in args if f in MODEL_FLAGS]
    inter_flag = [f for f in args if f in ("-v", "-w")]
    thr = ["-t", str(threads)] if threads > 0 else []
    if model or inter_flag:
        ngpred = args[args.index("-n") + 1] if "-n" in args else "1"
        rest = [f for f in args if f in ("-b", "-f", "-i")]
        fac = args[args.index(model[0]) + 1] if model and model[0] in ("-z", "-y") else "-"
        code = str(MODEL_FLAGS[model[0]]) if model else "-1"
        if inter_flag:
            rest += [inter_flag[0], args[args.index(inter_flag[0]) + 1]]
        return [REF_MODEL, pre + "XL", pre + "XR", pre + "Y", out, ngpred, code, fac] + rest + thr
    return [REF_BIN, "-c", pre + "XL", "-g", pre + "XR", "-p", pre + "Y", "-o", out] + args + thr


def main(only=None):
    """Run every case, or only the named ones (merged into the existing manifest)."""
    if not os.path.exists(REF_BIN):
        sys.exit("build the reference first: make -C oracle")
    manifest = {}
    if only:
        with open(os.path.join(HERE, "manifest.json")) as f:
            manifest = json.load(f)["cases"]
    tmp = tempfile.mkdtemp(prefix="oa_golden_")
    try:
        for case, (over, post, flagsets) in CASES.items():
            if only and case not in only:
                continue
            pre, extra = build_inputs(case, tmp)
            cdir = os.path.join(HERE, case)
            os.makedirs(cdir, exist_ok=True)
            entry = {"workload": over, "post": post, "inputs": input_digests(pre), "runs": {}}
            for flags in flagsets:
                tag = flag_tag(flags)
                out = os.path.join(tmp, f"{case}_{tag}")
                cmd = ref_command(flags, pre, extra, out)
                p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
                if p.returncode != 0:
                    raise RuntimeError(f"{case} {flags}: exit {p.returncode}\n{p.stdout[-2000:]}")
                sig = int(p.stdout.split("Number of Significant Results:")[1].split()[0])
                with open(out + "_dis.txt", "rb") as f, \
                        open(os.path.join(cdir, f"{tag}_dis.txt.gz"), "wb") as raw, \
                        gzip.GzipFile(fileobj=raw, mode="wb", mtime=0, filename="") as g:
                    shutil.copyfileobj(f, g)
                files = ["dis.txt.gz"]
                if "-b" in flags:
                    for ext in (("dbin",) if "-w" in flags else ("ibin", "dbin")):
                        shutil.copy(out + f"_sto.{ext}", os.path.join(cdir, f"{tag}_sto.{ext}"))
                        files.append(f"sto.{ext}")
                entry["runs"][tag] = {"flags": flags, "significant": sig, "files": files}
                print(f"{case:12s} {tag:10s} significant={sig}")
            manifest[case] = entry
        with open(os.path.join(HERE, "manifest.json"), "w") as f:
            json.dump({"exclude_list": EXCLUDE_LIST, "cases": manifest}, f, indent=1, sort_keys=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main(sys.argv[1:])
