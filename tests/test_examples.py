"""The reference's own shipped example data (examples/interactions, subset in
tests/golden/examples/ by make_examples.py) and the reference's outputs on it:
covariates with NaN values (their individuals dropped), NaN dosages (mean
imputed), missing phenotypes, the exclusion list, one set of interaction
columns (-v) and one analysis per interaction column (-w) with one random
column, two random columns (three columns per SNP) and a random plus an
all-zero column (singular systems: no results), and the additive dosage
model.  The phenotypes have missing values, so the reference's r >= 2
downdate applies: the oracle and the GPU run reproduce it (quirk mode).

* CPU: the FP64 oracle reproduces every golden row (same rows, names, n)
  within 1e-4 |t| + 1e-4 and the significant-result counts exactly;
* GPU: the CLI gives the same rows and counts within the same bar."""
import gzip
import json
import os
import subprocess
import tempfile

import pytest

import golden_util as GU
import oa_oracle as O
from omicabelnomm_b200 import engine as E

EX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "examples")
MANIFEST = json.load(open(os.path.join(EX, "manifest.json")))
T_REL, T_ABS = 1e-4, 1e-4


def _settings(run):
    flag, inter, ncol, model = run
    s = O.Settings()
    s.fname_excludelist = os.path.join(EX, "exclude_individuals.txt")
    s.fname_interactions = os.path.join(EX, inter)
    s.multi_interactions = flag == "-w"
    s.r = ncol
    if model == 0:
        s.model = 1          # additive
    s.quirk_r2 = True
    return s


def _golden(tag):
    with gzip.open(os.path.join(EX, f"{tag}_dis.txt.gz"), "rt") as f:
        tmp = tempfile.NamedTemporaryFile("w", suffix="_dis.txt", delete=False)
        tmp.write(f.read())
        tmp.close()
    try:
        return O.parse_dis(tmp.name)
    finally:
        os.unlink(tmp.name)


def _same_rows(ref, ours):
    assert [(r["Phe"], r["SNP"]) for r in ref] == [(r["Phe"], r["SNP"]) for r in ours], "rows or order differ"
    for a, b in zip(ref, ours):
        assert (a["n"], a["nPct"]) == (b["n"], b["nPct"])
        assert abs(a["T"] - b["T"]) <= T_REL * abs(a["T"]) + T_ABS, (a, b)
        assert abs(a["SE"] - b["SE"]) <= 2e-4 * abs(a["SE"]) + 1.5e-7, (a, b)


@pytest.mark.parametrize("tag", sorted(MANIFEST))
def test_oracle_matches_reference_on_its_example_data(tag):
    run = MANIFEST[tag]
    s = _settings(run["run"])
    res, inp = O.run_files(os.path.join(EX, "XL"), os.path.join(EX, "XR"), os.path.join(EX, "Y"), s,
                           keep_dense=True)
    _same_rows(_golden(tag), GU.oracle_rows(res, inp, s))
    assert res.total_sig == run["significant"]


@pytest.mark.gpu
@pytest.mark.parametrize("tag", sorted(MANIFEST))
def test_cli_matches_reference_on_its_example_data(tag, tmp_path):
    run = MANIFEST[tag]
    flag, inter, ncol, model = run["run"]
    out = str(tmp_path / "gpu")
    cmd = [E.CLI_PATH, "-c", os.path.join(EX, "XL"), "-g", os.path.join(EX, "XR"), "-p", os.path.join(EX, "Y"),
           "-o", out, "-x", os.path.join(EX, "exclude_individuals.txt"), flag, os.path.join(EX, inter),
           "--quirk-r2"] + (["-n", str(ncol)] if ncol > 1 else []) + (["-j"] if model == 0 else [])
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    sig = int(p.stdout.split("Number of Significant Results:")[1].split()[0])
    _same_rows(_golden(tag), O.parse_dis(out + "_dis.txt"))
    assert sig == run["significant"]
