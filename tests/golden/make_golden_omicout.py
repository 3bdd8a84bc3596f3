"""Generate the omicout fixtures: outputs of the reference's omicout on the
committed binary fixtures.

Run in a container where the reference tree is present and its omicout has
been compiled from its own source (``make -C oracle``):

    python tests/golden/make_golden_omicout.py

For every committed ``tests/golden/<case>/<tag>_sto.dbin`` (with its .ibin)
and every flag set in FLAGSETS, this runs ``oracle/_ref/omicout_ref`` and
stores its text output as ``tests/golden/<case>/<tag>_omicout_<flags>.txt.gz``;
``tests/golden/omicout_manifest.json`` lists the runs with their exit status
and row count.
"""
from __future__ import annotations

import glob
import gzip
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "omicout_ref")

# (name, flags): P and R2 thresholds, covariates, forced output
FLAGSETS = [
    ("p05", ["-d", "0.05"]),
    ("p001_r01", ["-d", "0.001", "-r", "0.01"]),
    ("p05_i", ["-d", "0.05", "-i"]),
    ("p05_f", ["-d", "0.05", "-f"]),
    ("p1", ["-d", "1"]),
    ("p2_i_r005", ["-d", "0.2", "-i", "-r", "0.005"]),
    ("f_i", ["-d", "0.5", "-f", "-i"]),
]


def main():
    if not os.path.exists(REF_BIN):
        sys.exit("build the reference first: make -C oracle")
    runs = {}
    tmp = tempfile.mkdtemp(prefix="oa_omicout_")
    try:
        for dbin in sorted(glob.glob(os.path.join(HERE, "*", "*_sto.dbin"))):
            base = dbin[: -len(".dbin")]
            case = os.path.basename(os.path.dirname(dbin))
            tag = os.path.basename(base)[: -len("_sto")]
            # the reference cuts -b at its first '.': hand it a dot-free copy
            src = os.path.join(tmp, f"{case}_{tag}_sto")
            for ext in (".ibin", ".dbin"):
                shutil.copy(base + ext, src + ext)
            for name, flags in FLAGSETS:
                out = os.path.join(tmp, "out")
                p = subprocess.run([REF_BIN, "-b", src, "-o", out] + flags, capture_output=True, text=True,
                                   timeout=300)
                key = f"{case}/{tag}_omicout_{name}"
                with open(out + ".txt", "rb") as f:
                    data = f.read()
                with open(os.path.join(HERE, key + ".txt.gz"), "wb") as raw, \
                        gzip.GzipFile(fileobj=raw, mode="wb", mtime=0, filename="") as g:
                    g.write(data)
                runs[key] = {"source": f"{case}/{tag}_sto", "flags": flags, "exit": p.returncode,
                             "rows": data.count(b"\n")}
                print(f"{key:40s} exit={p.returncode} rows={runs[key]['rows']}")
        with open(os.path.join(HERE, "omicout_manifest.json"), "w") as f:
            json.dump({"flagsets": dict(FLAGSETS), "runs": runs}, f, indent=1, sort_keys=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main()
