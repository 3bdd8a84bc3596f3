"""omicout (re-thresholding of the binary outputs) against the reference's own
omicout: the committed fixtures are its text output on the committed
.ibin/.dbin files of the reference CLI (tests/golden/make_golden_omicout.py);
ours must print the same bytes.  Host code only: no GPU needed."""
import gzip
import json
import os
import shutil
import struct
import subprocess

import pytest

from omicabelnomm_b200 import engine as E

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
MANIFEST = json.load(open(os.path.join(GOLDEN, "omicout_manifest.json")))
RUNS = sorted(MANIFEST["runs"])


def _source(tmp_path, key):
    """A dot-free copy of the run's .ibin/.dbin (the CLI cuts -b at its first '.')."""
    src = MANIFEST["runs"][key]["source"]
    dst = os.path.join(str(tmp_path), src.replace("/", "_"))
    for ext in (".ibin", ".dbin"):
        shutil.copy(os.path.join(GOLDEN, src + ext), dst + ext)
    return dst


def _expected(key):
    with gzip.open(os.path.join(GOLDEN, key + ".txt.gz"), "rb") as f:
        return f.read()


@pytest.mark.parametrize("key", RUNS)
def test_cli_prints_the_reference_bytes(tmp_path, key):
    run = MANIFEST["runs"][key]
    src = _source(tmp_path, key)
    out = os.path.join(str(tmp_path), "out")
    p = subprocess.run([E.OMICOUT_PATH, "-b", src, "-o", out] + run["flags"], capture_output=True, text=True,
                       timeout=120)
    assert p.returncode == run["exit"], p.stdout
    with open(out + ".txt", "rb") as f:
        got = f.read()
    assert got == _expected(key)


@pytest.mark.parametrize("key", [k for k in RUNS if k.endswith(("_p05", "_p05_i", "_f_i"))])
def test_library_call_matches_the_cli(tmp_path, key):
    run = MANIFEST["runs"][key]
    src = _source(tmp_path, key)
    f = run["flags"]
    min_p = float(f[f.index("-d") + 1])
    min_r2 = float(f[f.index("-r") + 1]) if "-r" in f else -100.0
    out = os.path.join(str(tmp_path), "lib_out")
    rows = E.omicout(src, out, min_p, min_r2, force_all="-f" in f, include_cov="-i" in f)
    with open(out + ".txt", "rb") as fh:
        got = fh.read()
    assert got == _expected(key)
    assert rows == run["rows"]


def test_missing_arguments_exit_1(tmp_path):
    key = RUNS[0]
    src = _source(tmp_path, key)
    p = subprocess.run([E.OMICOUT_PATH, "-b", src, "-o", os.path.join(str(tmp_path), "o")], capture_output=True,
                       text=True, timeout=60)
    assert p.returncode == 1 and "Missing arguments!" in p.stdout
    p = subprocess.run([E.OMICOUT_PATH, "-b", os.path.join(str(tmp_path), "absent"), "-o",
                        os.path.join(str(tmp_path), "o"), "-d", "0.05"], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1 and "Error reading File" in p.stdout


def test_invalid_info_file_exit_1(tmp_path):
    key = RUNS[0]
    src = _source(tmp_path, key)
    with open(src + ".ibin", "r+b") as f:        # l = 1: the reference refuses it
        f.seek(4)
        f.write(struct.pack("<i", 1))
    p = subprocess.run([E.OMICOUT_PATH, "-b", src, "-o", os.path.join(str(tmp_path), "o"), "-d", "0.05"],
                       capture_output=True, text=True, timeout=60)
    assert p.returncode == 1 and "invalid info data" in p.stdout
