"""Measure the reference's own numerical noise on every golden run.

Run where the reference CLI has been compiled from its own sources
(``make -C oracle``):

    python tests/golden/measure_noise.py

For every golden run this re-runs the reference at 1 and at 8 threads on the
regenerated inputs (the committed golden outputs were written at the
reference's default of 1 thread) and compares both with the FP64 oracle.
Per run it records, in ``tests/golden/noise.json``:

* ``dt_threads``: max |t_1 - t_8| over the rows both runs print - the spread
  of the reference against itself (its OpenMP/BLAS reduction orders);
* ``dt_fp64``: max |t_ref - t_fp64| of the golden (1-thread) rows against the
  FP64 restatement;
* ``dt_fp64_excess``: max (|t_ref - t_fp64| - 1e-4 |t_ref|), floored at 0 -
  how far the reference's FP32 answers sit from exact arithmetic beyond the
  relative part of the parity bar;
* ``dse_rel_fp64`` / ``dr2_fp64``: max relative SE and absolute R2
  deviation of the golden rows from the FP64 restatement;
* ``rows``: rows compared.

The parity bar of the GPU CLI against the golden outputs is then
|t - t_ref| <= 1e-4 |t_ref| + delta with delta = max(dt_threads,
dt_fp64_excess) + 1e-4 (the last term: the plain form's own absolute
allowance against FP64), see tests/golden_util.py.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

import golden_util as GU  # noqa: E402
import oa_oracle as O  # noqa: E402
from golden import make_golden as MG  # noqa: E402

QUIRK_RUNS = {("r2_missing", "nf"), ("r1_dosf", "nz"), ("r3_missing", "nf")}   # the reference's r >= 2 downdate applies


def _by_key(rows):
    return {(r["Phe"], r["SNP"]): r for r in rows}


def measure(case: str, tag: str, tmp: str) -> dict:
    pre, extra = GU.materialise(case, tmp)
    run = GU.manifest()["cases"][case]["runs"][tag]
    outs = {}
    for thr in (1, 8):
        out = os.path.join(tmp, f"{case}_{tag}_t{thr}")
        p = subprocess.run(MG.ref_command(run["flags"], pre, extra, out, threads=thr), capture_output=True,
                           text=True, timeout=600)
        if p.returncode != 0:
            raise RuntimeError(f"{case} {tag} -t {thr}: exit {p.returncode}\n{p.stdout[-2000:]}")
        outs[thr] = _by_key(O.parse_dis(out + "_dis.txt"))
    common = outs[1].keys() & outs[8].keys()
    dt_thr = max((abs(outs[1][k]["T"] - outs[8][k]["T"]) for k in common), default=0.0)
    s = GU.settings_for(run["flags"], extra)
    if (case, tag) in QUIRK_RUNS:
        s.quirk_r2 = True
    res, inp = O.run_files(pre + "XL", pre + "XR", pre + "Y", s, keep_dense=True)
    ours = _by_key(GU.oracle_rows(res, inp, s))
    ref = _by_key(GU.golden_rows(case, tag))
    both = ref.keys() & ours.keys()
    keys = sorted(both)

    def dev(field, rel):
        if not keys:
            return 0.0
        a = np.array([ref[k][field] for k in keys])
        b = np.array([ours[k][field] for k in keys])
        d = np.abs(a - b)
        return float((d / np.maximum(np.abs(a), 1e-30)).max() if rel else d.max())

    d = np.array([abs(ref[k]["T"] - ours[k]["T"]) for k in keys]) if keys else np.zeros(1)
    tr = np.array([abs(ref[k]["T"]) for k in keys]) if keys else np.zeros(1)
    return {"dt_threads": float(dt_thr), "dt_fp64": float(d.max()),
            "dt_fp64_excess": float(max(0.0, (d - 1e-4 * tr).max())), "dse_rel_fp64": dev("SE", True),
            "dr2_fp64": dev("R2", False), "rows": len(keys)}


def main():
    if not os.path.exists(MG.REF_BIN):
        sys.exit("build the reference first: make -C oracle")
    out = {}
    with tempfile.TemporaryDirectory(prefix="oa_noise_") as tmp:
        for case, tag in GU.all_runs():
            out.setdefault(case, {})[tag] = m = measure(case, tag, tmp)
            print(f"{case:12s} {tag:8s} threads {m['dt_threads']:.2e}  fp64 {m['dt_fp64']:.2e}  "
                  f"excess {m['dt_fp64_excess']:.2e}  se {m['dse_rel_fp64']:.1e}  r2 {m['dr2_fp64']:.1e}  "
                  f"rows {m['rows']}", flush=True)
    with open(os.path.join(HERE, "noise.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
