"""Measure the reference's own deviation from the FP64 oracle on the
quirk-mode dense test cases (tests/quirk_cases.py).

Run where the reference CLI has been compiled from its own sources
(``make -C oracle``):

    python tests/golden/measure_quirk_noise.py

Each case is written as .fvi/.fvd files and run through the reference CLI
with ``-f -n r`` (every result printed; the reference always applies its r >= 2
downdate, src/Algorithm.cpp:1300, 1390-1396); its rows are compared with the
oracle's quirk restatement (FP64).  Per case it records, in
``tests/golden/quirk_noise.json``, over the regular tests the reference prints:

* ``dse_rel``: max |SE_ref - SE_fp64| / SE_fp64;
* ``dr2``: max |R2_ref - R2_fp64| / max(|R2_fp64|, 1);
* ``dt_sys``: max |t_ref - t_fp64| / (the largest |t_fp64| of the test's SNP terms);
* ``rows``: rows compared.

The quirk's downdate can leave a system far from positive definite, so these
deviations grow with its condition number; the GPU tests hold the engine to
bars built from them.
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

import oa_oracle as O  # noqa: E402
import quirk_cases as QC  # noqa: E402
from golden import make_golden as MG  # noqa: E402
from omicabelnomm_b200 import synth  # noqa: E402


def measure(case: str, tmp: str) -> dict:
    r, ds = QC.build(case)
    pre = os.path.join(tmp, case + "_")
    synth.write_dataset(ds, pre)
    out = os.path.join(tmp, case + "_out")
    cmd = [MG.REF_BIN, "-c", pre + "XL", "-g", pre + "XR", "-p", pre + "Y", "-o", out, "-f", "-n", str(r)]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    if p.returncode != 0:
        raise RuntimeError(f"{case}: exit {p.returncode}\n{p.stdout[-2000:]}")
    ref = O.parse_dis(out + "_dis.txt")
    l, n = ds.XL.shape
    inp = O.Inputs(XL=ds.XL, XR=ds.XR, Y=ds.Y, xl_names=ds.xl_names, xr_names=ds.xr_names,
                   y_names=ds.y_names, realN=n, kept=np.arange(n))
    D = O.solve(inp, O.Settings(r=r, storePInd=True, quirk_r2=True), keep_dense=True).dense
    yidx = {name: j for j, name in enumerate(inp.y_names)}
    term = {" " + inp.xr_names[i * r + h]: (i, h) for i in range(len(inp.xr_names) // r) for h in range(r)}
    dse, dr2, dts = [], [], []
    for row in ref:
        if row["SNP"] not in term:      # covariate rows (-c display) are not SNP terms
            continue
        j = yidx[row["Phe"]]
        i, h = term[row["SNP"]]
        if D.singular[j, i]:
            continue
        se, r2, t = D.se[j, i, l + h], D.r2[j, i], D.tstat[j, i, l + h]
        dse.append(abs(row["SE"] - se) / abs(se))
        dr2.append(abs(row["R2"] - r2) / max(abs(r2), 1.0))
        dts.append(abs(row["T"] - t) / np.abs(D.tstat[j, i, l:]).max())
    return {"dse_rel": float(max(dse)), "dr2": float(max(dr2)), "dt_sys": float(max(dts)), "rows": len(dse)}


def main():
    if not os.path.exists(MG.REF_BIN):
        sys.exit("build the reference first: make -C oracle")
    out = {}
    with tempfile.TemporaryDirectory(prefix="oa_qnoise_") as tmp:
        for case in QC.CASES:
            out[case] = m = measure(case, tmp)
            print(f"{case:12s} se {m['dse_rel']:.2e}  r2 {m['dr2']:.2e}  t/tsys {m['dt_sys']:.2e}  rows {m['rows']}",
                  flush=True)
    with open(os.path.join(HERE, "quirk_noise.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
