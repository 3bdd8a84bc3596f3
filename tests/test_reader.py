"""The .fvi/.fvd reader of the CLI (the reference's AIOwrapper input path,
src/AIOwrapper.h:145-175, src/AIOwrapper.cpp:2294-2317, 1098-1130), hardened:

* float (type 5) and double (type 6) data files are read, integer types are
  refused with a message (the reference reads every file as float and never
  checks the type field);
* a truncated .fvi header or name table, and an .fvd shorter than its
  header's nobs x nvar values, are refused before any work starts;
* values are addressed with 64-bit file offsets, so a genotype file beyond
  2^31 values (the limit of the reference's int offsets,
  src/AIOwrapper.cpp:909-913, 1196) is read to its last SNP.

The refusals happen before the engine touches a GPU and run on CPU; reading
double files and files beyond 2^31 values runs a scan and needs a GPU.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

import oa_oracle as O
from omicabelnomm_b200 import engine as E
from omicabelnomm_b200 import fvformat, synth


def _dataset(where, seed=1, n=60, m=12, t=3):
    ds = synth.generate(synth.scaled(0, n=n, m=m, t=t, seed=seed))
    pre = os.path.join(where, "d_")
    synth.write_dataset(ds, pre)
    return ds, pre


def _cli(pre, out, *extra):
    cmd = [E.CLI_PATH, "-c", pre + "XL", "-g", pre + "XR", "-p", pre + "Y", "-o", out, *extra]
    return subprocess.run(cmd, capture_output=True, text=True, timeout=300)


def _set_type(fvi, type_code, bytes_per_record):
    raw = bytearray(open(fvi, "rb").read())
    struct.pack_into("<H", raw, 0, type_code)
    struct.pack_into("<I", raw, 16, bytes_per_record)
    struct.pack_into("<I", raw, 20, 8 * bytes_per_record)
    open(fvi, "wb").write(bytes(raw))


needs_cli = pytest.mark.skipif(not os.path.exists(E.CLI_PATH), reason="CLI not built")


@needs_cli
@pytest.mark.parametrize("type_code,nbytes", [(4, 4), (1, 2), (8, 1)])
def test_integer_types_are_refused(tmp_path, type_code, nbytes):
    _, pre = _dataset(str(tmp_path))
    _set_type(pre + "XR.fvi", type_code, nbytes)
    p = _cli(pre, str(tmp_path / "o"))
    assert p.returncode == 1
    assert f"data type {type_code}" in p.stdout + p.stderr


@needs_cli
def test_truncated_fvi_header_is_refused(tmp_path):
    _, pre = _dataset(str(tmp_path))
    raw = open(pre + "Y.fvi", "rb").read()
    open(pre + "Y.fvi", "wb").write(raw[:20])
    p = _cli(pre, str(tmp_path / "o"))
    assert p.returncode == 1 and "truncated header" in p.stdout + p.stderr


@needs_cli
def test_truncated_fvi_name_table_is_refused(tmp_path):
    _, pre = _dataset(str(tmp_path))
    raw = open(pre + "XL.fvi", "rb").read()
    open(pre + "XL.fvi", "wb").write(raw[:-5])
    p = _cli(pre, str(tmp_path / "o"))
    assert p.returncode == 1 and "name bytes" in p.stdout + p.stderr


@needs_cli
@pytest.mark.parametrize("which", ["XR", "Y", "XL"])
def test_short_fvd_is_refused_before_the_scan(tmp_path, which):
    _, pre = _dataset(str(tmp_path))
    raw = open(pre + which + ".fvd", "rb").read()
    open(pre + which + ".fvd", "wb").write(raw[:-4])
    p = _cli(pre, str(tmp_path / "o"))
    assert p.returncode == 1 and "truncated file" in p.stdout + p.stderr
    assert not os.path.exists(str(tmp_path / "o_dis.txt")) or os.path.getsize(str(tmp_path / "o_dis.txt")) == 0


def write_double(prefix, data, obs, names):
    """An .fvi/.fvd pair of DatABEL type 6 (double)."""
    fvformat.write_fv(prefix, data, obs, names)
    _set_type(prefix + ".fvi", 6, 8)
    np.ascontiguousarray(data, dtype=np.float64).tofile(prefix + ".fvd")


@pytest.mark.gpu
def test_double_files_give_the_float_results(tmp_path):
    ds, pre = _dataset(str(tmp_path), seed=5, n=300, m=80, t=6)
    a = _cli(pre, str(tmp_path / "f"), "-f")
    assert a.returncode == 0, a.stdout[-2000:]
    obs = fvformat.obs_names(ds.XL.shape[1])
    dpre = str(tmp_path / "dbl_")
    write_double(dpre + "XL", ds.XL, obs, ds.xl_names)
    write_double(dpre + "XR", ds.XR, obs, ds.xr_names)
    write_double(dpre + "Y", ds.Y, obs, ds.y_names)
    b = _cli(dpre, str(tmp_path / "d"), "-f")
    assert b.returncode == 0, b.stdout[-2000:]
    # the values are float32 numbers in both files: identical output
    assert open(str(tmp_path / "f_dis.txt")).read() == open(str(tmp_path / "d_dis.txt")).read()


@pytest.mark.gpu
def test_genotype_file_beyond_2_31_values(tmp_path):
    """A sparse XR file of 2,150,000 SNPs x 1,000 individuals (2.15e9 values, 8.6 GB
    apparent size): the last shard's SNPs, all beyond value 2^31, are read through
    64-bit offsets and give the results of a small file holding only them."""
    n, m_big = 1000, 2_150_000
    ds = synth.generate(synth.scaled(0, n=n, m=64, t=4, seed=9))
    pre = str(tmp_path / "big_")
    obs = fvformat.obs_names(n)
    fvformat.write_fv(pre + "XL", ds.XL, obs, ds.xl_names)
    fvformat.write_fv(pre + "Y", ds.Y, obs, ds.y_names)
    names = [f"snp{i}" for i in range(m_big)]
    fvformat.write_fv(pre + "XR", ds.XR[:1], obs, names[:1])          # header and names written below
    hdr = bytearray(open(pre + "XR.fvi", "rb").read(48))
    struct.pack_into("<I", hdr, 4, (n * m_big) & 0xFFFFFFFF)
    struct.pack_into("<I", hdr, 12, m_big)
    with open(pre + "XR.fvi", "wb") as f:
        f.write(bytes(hdr))
        for s in obs + names:
            b = s.encode()
            f.write(b + b"\0" * (32 - len(b)))
    shards, shard = 1000, 999          # the last shard: SNPs [999 * 2150, 2150000)
    first = shard * (m_big // shards)
    cnt = m_big - first
    assert first * n > 2 ** 31
    # the last shard's SNPs: the 64 real SNPs repeated; every other value is a hole (zeros)
    block = np.concatenate([ds.XR] * (cnt // 64 + 1))[:cnt]
    with open(pre + "XR.fvd", "wb") as f:
        f.truncate(4 * n * m_big)
        f.seek(4 * n * first)
        f.write(np.ascontiguousarray(block, dtype=np.float32).tobytes())
    a = _cli(pre, str(tmp_path / "big"), "-f", "--shard", f"{shard}/{shards}")
    assert a.returncode == 0, a.stdout[-2000:]
    small = str(tmp_path / "small_")
    fvformat.write_fv(small + "XL", ds.XL, obs, ds.xl_names)
    fvformat.write_fv(small + "Y", ds.Y, obs, ds.y_names)
    fvformat.write_fv(small + "XR", block, obs, names[first:])
    b = _cli(small, str(tmp_path / "sm"), "-f")
    assert b.returncode == 0, b.stdout[-2000:]
    big_rows = O.parse_dis(str(tmp_path / f"big_mpi{shard + 1}__dis.txt"))
    small_rows = O.parse_dis(str(tmp_path / "sm_dis.txt"))
    assert len(big_rows) == len(small_rows) == 4 * cnt
    for x, y in zip(big_rows, small_rows):
        assert (x["Phe"], x["SNP"], x["T"], x["B"], x["SE"]) == (y["Phe"], y["SNP"], y["T"], y["B"], y["SE"])
