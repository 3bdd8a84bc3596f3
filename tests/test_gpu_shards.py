"""SNP shards through the CLI (the reference's MPI mode, one process per
GPU): shard k of N writes <out>_mpi<k+1>__dis.txt (and _sto files) for its
SNP range; the shards' rows together are the unsharded run's rows, and each
shard's .ibin holds its own SNP count and names."""
import os
import struct
import subprocess

import pytest

import golden_util as GU
from omicabelnomm_b200 import engine as E

pytestmark = pytest.mark.gpu


def _cli(pre, out, extra_args, env=None):
    cmd = [E.CLI_PATH, "-c", pre + "XL", "-g", pre + "XR", "-p", pre + "Y", "-o", out, "-b"] + extra_args
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    return int(p.stdout.split("Number of Significant Results:")[1].split()[0])


def _rows(path):
    with open(path) as f:
        lines = f.read().splitlines()
    assert lines[0].startswith("Phe\tSNP")
    return lines[1:]


@pytest.mark.parametrize("via_env", [False, True])
def test_shards_cover_the_unsharded_run(tmp_path, via_env):
    pre, _ = GU.materialise("r1_tblocks", str(tmp_path))
    whole = str(tmp_path / "whole")
    sig_whole = _cli(pre, whole, [])
    rows_whole = _rows(whole + "_dis.txt")
    got, sig = [], 0
    m_total = 0
    for k in range(2):
        out = str(tmp_path / "sh")
        if via_env:   # launched by mpirun: rank and size from the environment
            env = dict(os.environ, OMPI_COMM_WORLD_RANK=str(k), OMPI_COMM_WORLD_SIZE="2")
            sig += _cli(pre, out, [], env=env)
        else:
            sig += _cli(pre, out, ["--shard", f"{k}/2"])
        base = f"{out}_mpi{k + 1}_"
        got += _rows(base + "_dis.txt")
        with open(base + "_sto.ibin", "rb") as f:
            n, l, r, t, m, namelen = struct.unpack("<6i", f.read(24))
        m_total += m
        assert os.path.getsize(base + "_sto.dbin") > 0
    with open(whole + "_sto.ibin", "rb") as f:
        m_whole = struct.unpack("<6i", f.read(24))[4]
    assert m_total == m_whole
    assert sorted(got) == sorted(rows_whole)
    assert sig == sig_whole
