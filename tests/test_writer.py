"""The CLI's host path (no GPU): its number formatting gives printf's characters, its parallel
formatting of stored rows gives the bytes of a plain sequential snprintf pass with the reference's
row format and .dbin records, and its parallel genotype reader returns the file's values
(tests/writer_check.cpp, compiled here against the host source with the engine calls stubbed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _cxx():
    return os.environ.get("CXX") or shutil.which("g++")


@pytest.mark.skipif(not _cxx() or not os.path.exists(os.path.join(CUDA, "include", "cuda_runtime.h")),
                    reason="needs g++ and the CUDA headers")
def test_writer_formats_like_printf(tmp_path):
    exe = str(tmp_path / "writer_check")
    src = os.path.join(ROOT, "tests", "writer_check.cpp")
    cmd = [_cxx(), "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(ROOT, "omicabelnomm_b200", "csrc"), "-I" + os.path.join(CUDA, "include"), src,
           "-o", exe, "-L" + os.path.join(CUDA, "lib64"), "-lcudart", "-lpthread"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    env = dict(os.environ, LD_LIBRARY_PATH=os.path.join(CUDA, "lib64") + ":" + os.environ.get("LD_LIBRARY_PATH", ""))
    p = subprocess.run([exe, "1000000"], capture_output=True, text=True, env=env, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "ok: 0 failures" in p.stdout
