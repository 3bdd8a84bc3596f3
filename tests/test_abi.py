"""The C ABI library: loads, exports what include/omicabel_b200.h declares,
and its host-only functions agree with the reference formulas (no GPU)."""
import ctypes as C
import math
import os
import subprocess

import numpy as np
import pytest

from omicabelnomm_b200 import engine as E
import oa_oracle as O


def test_library_exports_every_header_symbol():
    L = E.lib()
    syms = E.header_symbols()
    assert len(syms) >= 18
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert L.oa_abi_version() == 1


def test_struct_sizes_match_header():
    # field counts and packing of the public structs (all 4/8-byte fields)
    assert C.sizeof(E.Config) == 14 * 4
    assert C.sizeof(E.Rows) == 8 + 8 * 8 + 3 * 8
    assert C.sizeof(E.Outputs) == 8 * 5
    assert C.sizeof(E.Tuning) == 5 * 4


@pytest.mark.parametrize("p", [0.1, 0.05, 0.01, 1e-5, 5e-8])
def test_t_threshold_matches_oracle(p):
    assert abs(E.t_threshold(p) - float(O.thresholds(O.Settings(minPstore=p, minPdisp=0.0))[2])) < 2e-6


@pytest.mark.parametrize("t", [0.0, 0.7, 1.2834, 1.59, 1.6, 1.96, 3.5, 8.0, 30.0])
def test_pvalue_matches_reference_formula(t):
    tf = float(np.float32(t))
    assert E.pvalue(tf) == pytest.approx(O.pvalue(tf), rel=1e-12, abs=1e-300)


def test_pvalue_extreme_tail_is_long_double():
    # the reference prints P below 1e-308 (long double erfc), e.g. t = 133
    v = E.lib().oa_pvalue(C.c_float(133.0))
    assert 0.0 <= v < 1e-300 or v == 0.0


def test_cli_rejects_missing_arguments():
    p = subprocess.run([E.CLI_PATH], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1
    assert "Missing arguments" in p.stdout


def test_cli_rejects_unsupported_models():
    p = subprocess.run([E.CLI_PATH, "-j", "-c", "a", "-g", "b", "-p", "c", "-o", "d"], capture_output=True,
                       text=True, timeout=60)
    assert p.returncode == 1


def test_engine_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(E.OAError) as ei:
        E.Engine(100, 3, 1, 10, 10)
    assert ei.value.status == 2
    assert "CUDA" in str(ei.value) or "device" in str(ei.value)
