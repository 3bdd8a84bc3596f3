"""Golden fixtures from the reference's own shipped example data.

Run in a container where the reference tree is present and its CLI and
model driver have been compiled from its sources (``make -C oracle``):

    python tests/golden/make_examples.py

The reference's interaction tests (tests/test.cpp:188-311 of the reference)
run its solver on examples/interactions/{XL,XR,Y} - covariates with NaN
values, SNP columns with NaN dosages, phenotypes with missing values - with
the exclusion list examples/exclude_individuals.txt, limit_t = 50 traits and
limit_m = 100 SNP columns, and the interaction files INT*.  This script
copies a subset of that data into tests/golden/examples/ (the first 600
individuals, the first 50 traits, the first 100 SNP columns, the
interaction files the runs below use, the exclusion list) and records the
reference's outputs on it:

* -v (one set of interaction columns, the SNP column kept) and -w (one
  analysis per interaction column) with INTR (one random column), INTRR
  (two random columns: three columns per SNP) and INTR0 (a random and an
  all-zero column: the zero column makes its systems singular);
* the additive dosage model on two columns per SNP with -v INTR and -w INTRR.

The phenotypes have missing values, so the reference's r >= 2 downdate
applies to every run (the GPU runs them with --quirk-r2).  The runs go
through oracle/_ref/ref_model_driver, the reference's solver with the
interactions set in-process (its command line cannot reach them).
"""
from __future__ import annotations

import gzip
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from omicabelnomm_b200 import fvformat  # noqa: E402

REF_MODEL = os.path.join(ROOT, "oracle", "_ref", "ref_model_driver")
OUT = os.path.join(HERE, "examples")
N_IND, N_TRAITS, N_COLS = 600, 50, 100
INTER_FILES = ["INTR", "INTRR", "INTR0"]

# tag -> (interaction flag, interaction file, columns per SNP in the file, model code)
RUNS = {
    "v_R": ("-v", "INTR", 1, -1),
    "v_RR": ("-v", "INTRR", 1, -1),
    "v_R0": ("-v", "INTR0", 1, -1),
    "w_R": ("-w", "INTR", 1, -1),
    "w_RR": ("-w", "INTRR", 1, -1),
    "w_R0": ("-w", "INTR0", 1, -1),
    "add_v_R": ("-v", "INTR", 2, 0),
    "add_w_RR": ("-w", "INTRR", 2, 0),
}


def subset(src_dir: str) -> None:
    """The first N_IND individuals of every file, the first N_TRAITS traits and N_COLS SNP columns."""
    os.makedirs(OUT, exist_ok=True)
    for name, nvar in [("XL", None), ("XR", N_COLS), ("Y", N_TRAITS)] + [(f, None) for f in INTER_FILES]:
        hdr, obs, var = fvformat.read_fvi(os.path.join(src_dir, name))
        v = hdr.num_variables if nvar is None else min(nvar, hdr.num_variables)
        data = fvformat.read_fvd(os.path.join(src_dir, name), hdr.num_observations, hdr.num_variables, 0, v)
        fvformat.write_fv(os.path.join(OUT, name), np.ascontiguousarray(data[:, :N_IND]), obs[:N_IND], var[:v])
    shutil.copy(os.path.join(os.path.dirname(src_dir), "exclude_individuals.txt"),
                os.path.join(OUT, "exclude_individuals.txt"))


def ref_command(tag: str, out: str, threads: int = 0):
    flag, inter, ncol, model = RUNS[tag]
    cmd = [REF_MODEL, os.path.join(OUT, "XL"), os.path.join(OUT, "XR"), os.path.join(OUT, "Y"), out, str(ncol),
           str(model), "-", flag, os.path.join(OUT, inter), "-x", os.path.join(OUT, "exclude_individuals.txt")]
    return cmd + (["-t", str(threads)] if threads else [])


def main():
    ref = os.environ.get("OA_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))
    src = os.path.join(ref, "examples", "interactions")
    if not os.path.isdir(src) or not os.path.exists(REF_MODEL):
        sys.exit("needs the reference tree (OA_REFERENCE_DIR) and make -C oracle")
    subset(src)
    manifest = {}
    with tempfile.TemporaryDirectory(prefix="oa_examples_") as tmp:
        for tag in RUNS:
            out = os.path.join(tmp, tag)
            p = subprocess.run(ref_command(tag, out), capture_output=True, text=True, timeout=600)
            if p.returncode != 0:
                raise RuntimeError(f"{tag}: exit {p.returncode}\n{p.stdout[-2000:]}")
            sig = int(p.stdout.split("Number of Significant Results:")[1].split()[0])
            with open(out + "_dis.txt", "rb") as f, open(os.path.join(OUT, f"{tag}_dis.txt.gz"), "wb") as raw, \
                    gzip.GzipFile(fileobj=raw, mode="wb", mtime=0, filename="") as g:
                shutil.copyfileobj(f, g)
            manifest[tag] = {"run": list(RUNS[tag]), "significant": sig}
            print(f"{tag:10s} significant={sig}")
    with open(os.path.join(OUT, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
