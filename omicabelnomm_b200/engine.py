"""ctypes binding of the C ABI (include/omicabel_b200.h).

The library is the only compute path: if ``lib/libomicabel_b200.so`` is
missing, importing the functions raises instead of falling back to anything.
Build it with ``python -m omicabelnomm_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from dataclasses import dataclass
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libomicabel_b200.so")
CLI_PATH = os.path.join(HERE, "lib", "omicabelnomm")
OMICOUT_PATH = os.path.join(HERE, "lib", "omicout")
HEADER = os.path.join(os.path.dirname(HERE), "include", "omicabel_b200.h")

OA_OK = 0
STATUS = {0: "OA_OK", 1: "OA_ERR_ARG", 2: "OA_ERR_CUDA", 3: "OA_ERR_COLLINEAR", 4: "OA_ERR_IO",
          5: "OA_ERR_STATE", 6: "OA_ERR_NOMEM", 7: "OA_ERR_UNSUPPORTED", 8: "OA_ERR_NUMERIC"}
PLAIN, MIXED = 0, 1
# per-test status bits of Engine.dense_flags (OA_TEST_* in include/omicabel_b200.h)
TEST_SINGULAR, TEST_RSS, TEST_R2, TEST_STORED = 1, 2, 4, 8


class OAError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Config(C.Structure):
    _fields_ = [("n", C.c_int32), ("l", C.c_int32), ("r", C.c_int32), ("max_traits", C.c_int32),
                ("max_snps", C.c_int32), ("precision", C.c_int32), ("device", C.c_int32),
                ("disp_cov", C.c_int32), ("store_all", C.c_int32), ("quirk_r2", C.c_int32),
                ("min_r2_store", C.c_float), ("min_t_store", C.c_float), ("min_p_disp", C.c_float),
                ("real_n", C.c_int32)]


class Rows(C.Structure):
    _fields_ = [("count", C.c_int64), ("trait", C.POINTER(C.c_int32)), ("snp", C.POINTER(C.c_int32)),
                ("r2", C.POINTER(C.c_float)), ("n_used", C.POINTER(C.c_int32)),
                ("coef_mask", C.POINTER(C.c_uint32)), ("coef_b", C.POINTER(C.c_float)),
                ("coef_se", C.POINTER(C.c_float)), ("coef_t", C.POINTER(C.c_float)),
                ("sig_cov_unrowed", C.c_int64), ("tests", C.c_int64), ("singular", C.c_int64)]


class Settings(C.Structure):
    _fields_ = [("fname_xl", C.c_char_p), ("fname_xr", C.c_char_p), ("fname_y", C.c_char_p),
                ("fname_out", C.c_char_p), ("fname_exclude", C.c_char_p), ("r", C.c_int32),
                ("min_p_disp", C.c_float), ("min_p_store", C.c_float), ("min_r2_disp", C.c_float),
                ("min_r2_store", C.c_float), ("store_bin", C.c_int32), ("disp_cov", C.c_int32),
                ("store_all", C.c_int32), ("precision", C.c_int32), ("device", C.c_int32),
                ("quirk_r2", C.c_int32), ("verbose", C.c_int32), ("shard", C.c_int32), ("shards", C.c_int32),
                ("dosage_model", C.c_int32), ("fname_factors", C.c_char_p), ("fname_interactions", C.c_char_p),
                ("multi_interactions", C.c_int32)]


class Tuning(C.Structure):
    _fields_ = [("chunk_snps", C.c_int32), ("gemm_variant", C.c_int32), ("gemm_raster", C.c_int32),
                ("stats_path", C.c_int32), ("lean_spb", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class Outputs(C.Structure):
    _fields_ = [("total_sig_results", C.c_uint64), ("duration_s", C.c_double), ("tests", C.c_int64),
                ("rows_written", C.c_int64), ("singular", C.c_int64)]


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Load the engine library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m omicabelnomm_b200.build`")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    fp = C.POINTER(C.c_float)
    sig = {
        "oa_engine_create": ([C.POINTER(Config), C.POINTER(P)], C.c_int),
        "oa_engine_destroy": ([P], C.c_int),
        "oa_set_covariates": ([P, fp], C.c_int),
        "oa_set_traits": ([P, fp, C.c_int32], C.c_int),
        "oa_set_traits_device": ([P, P, C.c_int32], C.c_int),
        "oa_run_snps": ([P, fp, C.c_int32, C.POINTER(Rows)], C.c_int),
        "oa_run_snps_device": ([P, P, C.c_int32, C.c_int32, C.POINTER(Rows)], C.c_int),
        "oa_dense_last": ([P, fp, fp, fp, fp], C.c_int),
        "oa_enable_dense": ([P, C.c_int32], C.c_int),
        "oa_dense_flags": ([P, C.POINTER(C.c_uint8)], C.c_int),
        "oa_kernel_launches": ([P], C.c_int64),
        "oa_last_kernel_ms": ([P, C.POINTER(C.c_char_p)], C.c_float),
        "oa_last_stats_ms": ([P], C.c_float),
        "oa_last_block_ms": ([P], C.c_float),
        "oa_default_settings": ([C.POINTER(Settings)], None),
        "oa_solve": ([C.POINTER(Settings), C.POINTER(Outputs)], C.c_int),
        "oa_cli_main": ([C.c_int, C.POINTER(C.c_char_p)], C.c_int),
        "oa_pvalue": ([C.c_float], C.c_longdouble),
        "oa_t_threshold": ([C.c_float], C.c_float),
        "oa_last_error": ([], C.c_char_p),
        "oa_abi_version": ([], C.c_int32),
        "oa_scan_dense_noalloc": ([P, P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P, P, P, P,
                                   P], C.c_int),
        "oa_set_tuning": ([P, C.POINTER(Tuning)], C.c_int),
        "oa_shard_range": ([C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
        "oa_set_snp_rows": ([P, C.POINTER(C.c_int32), C.c_int32, C.c_int64], C.c_int),
        "oa_device_bytes": ([P], C.c_int64),
        "oa_reserve": ([P, C.c_int32, C.c_int32], C.c_int),
        "oa_set_column_model": ([P, C.c_int32, fp, C.c_int32], C.c_int),
        "oa_set_interactions": ([P, fp, C.c_int32, C.c_int32], C.c_int),
        "oa_omicout": ([C.c_char_p, C.c_char_p, C.c_float, C.c_float, C.c_int32, C.c_int32,
                        C.POINTER(C.c_int64)], C.c_int),
        "oa_omicout_main": ([C.c_int, C.POINTER(C.c_char_p)], C.c_int),
        "oa_get_tuning": ([P, C.POINTER(Tuning)], C.c_int),
        "oa_autotune": ([P, P, C.c_int32, C.POINTER(Tuning)], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def header_symbols() -> list[str]:
    """Every function the public header declares."""
    src = open(HEADER).read()
    decl = re.compile(r"^\s*(?:const\s+)?(?:oa_status|void|int|int32_t|int64_t|float|long double|char)\s*\**\s*"
                      r"(oa_[a-z0-9_]+)\s*\(", re.M)
    return sorted(set(decl.findall(src)))


def _check(st: int):
    if st != OA_OK:
        raise OAError(st, lib().oa_last_error().decode(errors="replace"))


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


@dataclass
class StoredRows:
    trait: np.ndarray
    snp: np.ndarray
    r2: np.ndarray
    n_used: np.ndarray
    mask: np.ndarray
    B: np.ndarray      # (count, p)
    SE: np.ndarray
    T: np.ndarray
    tests: int
    singular: int
    sig_cov_unrowed: int


class Engine:
    """One engine on one device (≙ one solver instance of the reference)."""

    def __init__(self, n: int, l: int, r: int, max_traits: int, max_snps: int, *, precision: int = PLAIN,
                 device: int = 0, disp_cov: bool = False, store_all: bool = False,
                 min_r2_store: float = 1e-6, min_t_store: Optional[float] = None, min_p_disp: float = 0.05,
                 real_n: Optional[int] = None, quirk_r2: bool = False):
        L = lib()
        if min_t_store is None:
            min_t_store = float(L.oa_t_threshold(C.c_float(0.1)))
        self.cfg = Config(n, l, r, max_traits, max_snps, precision, device, int(disp_cov), int(store_all),
                          int(quirk_r2), min_r2_store, min_t_store, min_p_disp, real_n or n)
        self.n, self.l, self.r, self.p = n, l, r, l + r
        h = C.c_void_p()
        _check(L.oa_engine_create(C.byref(self.cfg), C.byref(h)))
        self.h = h
        self.t = 0

    def close(self):
        if getattr(self, "h", None):
            lib().oa_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_covariates(self, XL: np.ndarray):
        """XL as a (l, n) float32 array (column-major n x l)."""
        XL = np.ascontiguousarray(XL, dtype=np.float32)
        assert XL.shape == (self.l, self.n)
        _check(lib().oa_set_covariates(self.h, _fptr(XL)))

    def set_traits(self, Y: np.ndarray):
        """Y as a (t, n) float32 array, NaN = missing."""
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        assert Y.shape[1] == self.n
        _check(lib().oa_set_traits(self.h, _fptr(Y), Y.shape[0]))
        self.t = Y.shape[0]

    def set_traits_device(self, ptr: int, t: int):
        _check(lib().oa_set_traits_device(self.h, C.c_void_p(ptr), t))
        self.t = t

    def enable_dense(self, on: bool = True):
        _check(lib().oa_enable_dense(self.h, int(on)))

    def run(self, XR: np.ndarray) -> StoredRows:
        """XR as a (mb*r, n) float32 array; returns the stored rows in (trait, SNP) order."""
        XR = np.ascontiguousarray(XR, dtype=np.float32)
        cols = getattr(self, "in_cols", 0) or self.r
        assert XR.shape[1] == self.n and XR.shape[0] % cols == 0
        rows = Rows()
        _check(lib().oa_run_snps(self.h, _fptr(XR), XR.shape[0] // cols, C.byref(rows)))
        return self._rows(rows)

    def run_raw(self, XR: np.ndarray) -> Rows:
        """Like run() but returns the C struct (host pointers owned by the engine, no copies)."""
        assert XR.dtype == np.float32 and XR.flags.c_contiguous and XR.shape[1] == self.n
        rows = Rows()
        _check(lib().oa_run_snps(self.h, _fptr(XR), XR.shape[0] // self.r, C.byref(rows)))
        return rows

    def run_device(self, ptr: int, mb: int, results_on_host: bool = False) -> Rows:
        rows = Rows()
        _check(lib().oa_run_snps_device(self.h, C.c_void_p(ptr), mb, int(results_on_host), C.byref(rows)))
        return rows

    def scan(self, ptr: int, mb: int) -> StoredRows:
        """Device SNP block -> stored rows on the host, in (trait, SNP) order (copied)."""
        return self._rows(self.run_device(ptr, mb, results_on_host=True))

    def _rows(self, rows: Rows) -> StoredRows:
        N, p = rows.count, self.p

        def arr(ptr, shape, dt):
            if N == 0:
                return np.zeros(shape, dtype=dt)
            return np.ctypeslib.as_array(ptr, shape=shape).astype(dt, copy=True)

        return StoredRows(trait=arr(rows.trait, (N,), np.int32), snp=arr(rows.snp, (N,), np.int32),
                          r2=arr(rows.r2, (N,), np.float32), n_used=arr(rows.n_used, (N,), np.int32),
                          mask=arr(rows.coef_mask, (N,), np.uint32), B=arr(rows.coef_b, (N, p), np.float32),
                          SE=arr(rows.coef_se, (N, p), np.float32), T=arr(rows.coef_t, (N, p), np.float32),
                          tests=rows.tests, singular=rows.singular, sig_cov_unrowed=rows.sig_cov_unrowed)

    def dense(self, mb: int):
        """beta/se/t (t, mb, r) and R2 (t, mb) of the last SNP block (needs enable_dense)."""
        t, r = self.t, self.r
        b = np.empty((t, mb, r), np.float32)
        se = np.empty_like(b)
        tt = np.empty_like(b)
        r2 = np.empty((t, mb), np.float32)
        _check(lib().oa_dense_last(self.h, _fptr(b), _fptr(se), _fptr(tt), _fptr(r2)))
        return b, se, tt, r2

    def dense_flags(self, mb: int) -> np.ndarray:
        """Per-test status bits (t, mb) of the last SNP block: TEST_SINGULAR, TEST_RSS, TEST_R2,
        TEST_STORED (0 = evaluated, nothing stored); needs enable_dense."""
        f = np.empty((self.t, mb), np.uint8)
        _check(lib().oa_dense_flags(self.h, f.ctypes.data_as(C.POINTER(C.c_uint8))))
        return f

    def set_tuning(self, **fields):
        """oa_set_tuning: chunk_snps, gemm_variant, gemm_raster, stats_path, lean_spb (0 = automatic)."""
        t = Tuning(**{k: int(v) for k, v in fields.items()})
        _check(lib().oa_set_tuning(self.h, C.byref(t)))

    def tuning(self) -> dict:
        t = Tuning()
        _check(lib().oa_get_tuning(self.h, C.byref(t)))
        return t.as_dict()

    def autotune(self, ptr: int, mb: int) -> dict:
        """oa_autotune on a device SNP block of mb SNPs; returns the tuning kept."""
        t = Tuning()
        _check(lib().oa_autotune(self.h, C.c_void_p(ptr), mb, C.byref(t)))
        return t.as_dict()

    def set_snp_rows(self, rows: Optional[np.ndarray], ld: int = 0):
        """Read device SNP columns of ``ld`` floats and use rows ``rows`` (ascending, n of them)."""
        if rows is None:
            _check(lib().oa_set_snp_rows(self.h, None, 0, 0))
            return
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        _check(lib().oa_set_snp_rows(self.h, rows.ctypes.data_as(C.POINTER(C.c_int32)), rows.size, ld))

    def device_bytes(self) -> int:
        return int(lib().oa_device_bytes(self.h))

    def set_column_model(self, in_cols: int, weights=None, combine: bool = True) -> None:
        """oa_set_column_model: SNPs arrive as in_cols file columns combined (or scaled) on the device."""
        w = np.ascontiguousarray(weights if weights is not None else np.ones(max(in_cols, 1)), dtype=np.float32)
        _check(lib().oa_set_column_model(self.h, int(in_cols), _fptr(w), int(combine)))
        self.in_cols = int(in_cols)

    def set_interactions(self, inter: np.ndarray, keep: bool = True) -> None:
        """oa_set_interactions: inter (k, n) float32; SNP column x -> [I_1 x, ..., I_k x (, x)]."""
        inter = np.ascontiguousarray(inter, dtype=np.float32)
        _check(lib().oa_set_interactions(self.h, _fptr(inter), inter.shape[0], int(keep)))
        if not getattr(self, "in_cols", 0):
            self.in_cols = 1

    def reserve(self, traits: int, snps: int) -> None:
        """oa_reserve: allocate now what blocks of up to `traits` traits x `snps` SNPs need."""
        _check(lib().oa_reserve(self.h, int(traits), int(snps)))

    def launches(self) -> int:
        return int(lib().oa_kernel_launches(self.h))

    def last_stats_ms(self) -> float:
        return float(lib().oa_last_stats_ms(self.h))

    def last_block_ms(self) -> float:
        """Device time of the last SNP block (CUDA events on the engine's stream)."""
        return float(lib().oa_last_block_ms(self.h))

    def last_kernel_ms(self):
        name = C.c_char_p()
        ms = lib().oa_last_kernel_ms(self.h, C.byref(name))
        return float(ms), (name.value or b"").decode()


def scan_dense_noalloc(xl_ptr: int, y_ptr: int, xr_ptr: int, n: int, l: int, r: int, t: int, mb: int,
                       beta_ptr: int, se_ptr: int, t_ptr: int, r2_ptr: int, stream: int = 0) -> None:
    """oa_scan_dense_noalloc on device pointers (see include/omicabel_b200.h)."""
    V = C.c_void_p
    _check(lib().oa_scan_dense_noalloc(V(xl_ptr), V(y_ptr), V(xr_ptr), n, l, r, t, mb, V(beta_ptr), V(se_ptr),
                                       V(t_ptr), V(r2_ptr), V(stream)))


def omicout(source: str, dest: str, min_p_disp: float, min_r2: float = -100.0, force_all: bool = False,
            include_cov: bool = False) -> int:
    """oa_omicout: <source>.ibin/.dbin -> <dest>.txt re-thresholded; returns the rows written."""
    rows = C.c_int64()
    _check(lib().oa_omicout(source.encode(), dest.encode(), C.c_float(min_p_disp), C.c_float(min_r2),
                            int(force_all), int(include_cov), C.byref(rows)))
    return rows.value


def shard_range(m: int, shard: int, shards: int) -> tuple[int, int]:
    """(first SNP, SNP count) of a shard: the reference's MPI split of m SNPs."""
    first, count = C.c_int32(), C.c_int32()
    _check(lib().oa_shard_range(m, shard, shards, C.byref(first), C.byref(count)))
    return first.value, count.value


def t_threshold(p: float) -> float:
    return float(lib().oa_t_threshold(C.c_float(p)))


def pvalue(t: float) -> float:
    return float(lib().oa_pvalue(C.c_float(t)))


def solve(xl: str, xr: str, y: str, out: str, *, r: int = 1, exclude: str = "", store_bin=False,
          disp_cov=False, store_all=False, precision=PLAIN, device=0, min_p_disp=None, min_p_store=None,
          min_r2_disp=None, min_r2_store=None, verbose=False, shard=0, shards=1, dosage_model=0,
          factors: str = "", interactions: str = "", multi_interactions=False) -> Outputs:
    """≙ Algorithm::solve on files: writes out_dis.txt (+ _sto.ibin/.dbin)."""
    L = lib()
    s = Settings()
    L.oa_default_settings(C.byref(s))
    keep = [v.encode() for v in (xl, xr, y, out, exclude, factors, interactions)]
    s.dosage_model = int(dosage_model)
    s.fname_factors = keep[5] if factors else None
    s.fname_interactions = keep[6] if interactions else None
    s.multi_interactions = int(bool(multi_interactions))
    s.fname_xl, s.fname_xr, s.fname_y, s.fname_out = keep[:4]
    s.fname_exclude = keep[4] if exclude else None
    s.r = r
    s.store_bin, s.disp_cov, s.store_all = int(store_bin), int(disp_cov), int(store_all)
    s.precision, s.device, s.verbose = precision, device, int(verbose)
    s.shard, s.shards = shard, shards
    if min_p_disp is not None:
        s.min_p_disp = min_p_disp
    if min_p_store is not None:
        s.min_p_store = min_p_store
    if min_r2_disp is not None:
        s.min_r2_disp = min_r2_disp
    if min_r2_store is not None:
        s.min_r2_store = min_r2_store
    o = Outputs()
    _check(L.oa_solve(C.byref(s), C.byref(o)))
    return o
