"""DatABEL filevector (.fvi/.fvd) reading and writing.

Layout (reference: src/AIOwrapper.h:145-175, reader src/AIOwrapper.cpp:2294-2317):

* ``.fvi`` — a 48-byte header: ``u16 type`` + 2 pad bytes, then the u32
  fields ``nelements, numObservations, numVariables, bytesPerRecord,
  bitsPerRecord, namelength`` and ``reserved[5]``.  It is followed by
  ``(numObservations + numVariables) * namelength`` name bytes: the
  observation (individual) names first, then the variable names, each
  NUL-padded to ``namelength``.
* ``.fvd`` — raw little-endian float32, variable-major: the
  ``numObservations`` values of variable 0, then variable 1, ...  The
  reference never checks ``type`` and always reads float32
  (src/AIOwrapper.cpp:1103-1125); this module does the same on read and
  writes ``type = 5`` (FLOAT_TYPE, src/AIOwrapper.h:145-152).  ``nelements``
  is a 32-bit field: files of 2^32 values or more store it modulo 2^32
  (readers size the data from ``numObservations * numVariables``).

Arrays in this package keep the file's variable-major order: a block of
``v`` variables over ``n`` observations is a C-contiguous ``(v, n)``
float32 array, i.e. the column-major ``n x v`` matrix the engine uses.
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

FVI_HEADER = struct.Struct("<H2xIIIIII5I")
assert FVI_HEADER.size == 48
FLOAT_TYPE = 5
DEFAULT_NAMELENGTH = 32


@dataclass
class FviHeader:
    type: int
    nelements: int
    num_observations: int
    num_variables: int
    bytes_per_record: int
    bits_per_record: int
    namelength: int
    reserved: tuple = field(default=(0, 0, 0, 0, 0))


def _strip(raw: bytes) -> str:
    """Names end at the first NUL, as ``string(&fvi_data[idx])`` reads them."""
    cut = raw.find(b"\0")
    return (raw if cut < 0 else raw[:cut]).decode("latin-1")


def read_fvi(prefix: str):
    """Return (header, observation names, variable names) of ``prefix.fvi``."""
    with open(prefix + ".fvi", "rb") as f:
        raw = f.read()
    if len(raw) < FVI_HEADER.size:
        raise ValueError(f"{prefix}.fvi: truncated header ({len(raw)} bytes)")
    vals = FVI_HEADER.unpack_from(raw, 0)
    hdr = FviHeader(vals[0], vals[1], vals[2], vals[3], vals[4], vals[5], vals[6],
                    tuple(vals[7:12]))
    nl = hdr.namelength
    body = raw[FVI_HEADER.size:]
    need = (hdr.num_observations + hdr.num_variables) * nl
    if len(body) < need:
        raise ValueError(f"{prefix}.fvi: {len(body)} name bytes, header needs {need}")
    obs = [_strip(body[i * nl:(i + 1) * nl]) for i in range(hdr.num_observations)]
    off = hdr.num_observations * nl
    var = [_strip(body[off + i * nl: off + (i + 1) * nl]) for i in range(hdr.num_variables)]
    return hdr, obs, var


def read_fvd(prefix: str, num_observations: int, num_variables: int,
             first_var: int = 0, count: int | None = None) -> np.ndarray:
    """Read variables ``[first_var, first_var+count)`` as a (count, n) float32 array."""
    if count is None:
        count = num_variables - first_var
    n = num_observations
    out = np.fromfile(prefix + ".fvd", dtype="<f4", count=count * n,
                      offset=first_var * n * 4)
    if out.size != count * n:
        raise ValueError(f"{prefix}.fvd: short read ({out.size} of {count * n} floats)")
    return out.reshape(count, n)


def _pack_names(names: Sequence[str], namelength: int) -> bytes:
    out = bytearray()
    for s in names:
        b = s.encode("latin-1")
        if len(b) >= namelength:
            raise ValueError(f"name {s!r} does not fit namelength {namelength}")
        out += b + b"\0" * (namelength - len(b))
    return bytes(out)


def write_fv(prefix: str, data: np.ndarray, obs_names: Sequence[str],
             var_names: Sequence[str], namelength: int = DEFAULT_NAMELENGTH) -> None:
    """Write a (num_variables, n) float32 array as ``prefix.fvi`` + ``prefix.fvd``."""
    data = np.ascontiguousarray(data, dtype="<f4")
    v, n = data.shape
    if len(obs_names) != n or len(var_names) != v:
        raise ValueError("name counts do not match the data shape")
    hdr = FVI_HEADER.pack(FLOAT_TYPE, (v * n) & 0xFFFFFFFF, n, v, 4, 32, namelength, 0, 0, 0, 0, 0)
    os.makedirs(os.path.dirname(os.path.abspath(prefix)), exist_ok=True)
    with open(prefix + ".fvi", "wb") as f:
        f.write(hdr)
        f.write(_pack_names(obs_names, namelength))
        f.write(_pack_names(var_names, namelength))
    data.tofile(prefix + ".fvd")


def write_fvd_chunked(prefix: str, n: int, var_names: Sequence[str],
                      obs_names: Sequence[str], chunks, namelength: int = DEFAULT_NAMELENGTH) -> None:
    """Write a large file from an iterator of (v_chunk, n) float32 blocks."""
    v = len(var_names)
    hdr = FVI_HEADER.pack(FLOAT_TYPE, (v * n) & 0xFFFFFFFF, n, v, 4, 32, namelength, 0, 0, 0, 0, 0)
    with open(prefix + ".fvi", "wb") as f:
        f.write(hdr)
        f.write(_pack_names(obs_names, namelength))
        f.write(_pack_names(var_names, namelength))
    written = 0
    with open(prefix + ".fvd", "wb") as f:
        for blk in chunks:
            blk = np.ascontiguousarray(blk, dtype="<f4")
            if blk.shape[1] != n:
                raise ValueError("chunk has the wrong number of observations")
            blk.tofile(f)
            written += blk.shape[0]
    if written != v:
        raise ValueError(f"wrote {written} variables, header says {v}")


def obs_names(n: int) -> List[str]:
    return [f"id{i + 1}" for i in range(n)]
