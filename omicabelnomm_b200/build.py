"""Build the engine library and CLI in-tree for sm_100a.

    python -m omicabelnomm_b200.build [-j N] [--force]

Products (git-ignored, they travel with the tree):
    omicabelnomm_b200/lib/libomicabel_b200.so   the C-ABI library (include/omicabel_b200.h)
    omicabelnomm_b200/lib/omicabelnomm          the CLI
    omicabelnomm_b200/lib/omicout               the re-thresholding tool for the binary outputs
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib")
OBJ = os.path.join(OUT, "obj")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["oa_engine.cu", "oa_stats.cu", "oa_gemm_simt.cu", "oa_gemm_tc.cu", "oa_noalloc.cu"]
CXX_SOURCES = ["oa_host.cpp", "oa_omicout.cpp"]
LIB = os.path.join(OUT, "libomicabel_b200.so")
CLI = os.path.join(OUT, "omicabelnomm")
OMICOUT = os.path.join(OUT, "omicout")


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    # the image's default CXX may lack OpenMP/spec files; the system g++ is complete
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _digest(paths) -> str:
    h = hashlib.sha256()
    for p in sorted(paths):
        with open(p, "rb") as f:
            h.update(p.encode() + f.read())
    return h.hexdigest()[:16]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "omicabel_b200.h"))
    return hs


def _compile(src: str, verbose: bool) -> str:
    path = os.path.join(CSRC, src)
    key = _digest([path] + _headers())
    obj = os.path.join(OBJ, f"{src}.{key}.o")
    if os.path.exists(obj):
        return obj
    common = ["-I" + INCLUDE, "-I" + CSRC]
    if src.endswith(".cu"):
        cmd = [nvcc(), "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", host_cxx(),
               "--expt-relaxed-constexpr", *common, "-c", path, "-o", obj + ".tmp"]
    else:
        cmd = [host_cxx(), "-std=c++17", "-O2", "-fPIC", "-I/usr/local/cuda/include", *common, "-c", path,
               "-o", obj + ".tmp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(obj + ".tmp", obj)
    return obj


def build(jobs: int = 0, verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    if force:
        for f in os.listdir(OBJ):
            os.unlink(os.path.join(OBJ, f))
    srcs = CU_SOURCES + CXX_SOURCES
    with cf.ThreadPoolExecutor(max_workers=jobs or len(srcs)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    cudalib = "/usr/local/cuda/lib64"
    link = [nvcc(), *ARCH, "-shared", "-ccbin", host_cxx(), "-o", LIB + ".tmp", *objs,
            "-L" + cudalib, "-lcudart", "-Xlinker", "-rpath," + cudalib]
    subprocess.run(link, check=True)
    os.replace(LIB + ".tmp", LIB)
    mains = []
    for src, exe in (("oa_cli.cpp", CLI), ("oa_omicout_cli.cpp", OMICOUT)):
        obj = _compile(src, verbose)
        subprocess.run([host_cxx(), "-o", exe + ".tmp", obj, "-L" + OUT, "-lomicabel_b200",
                        "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + cudalib, "-L" + cudalib, "-lcudart"], check=True)
        os.replace(exe + ".tmp", exe)
        mains.append(obj)
    # drop stale objects of older source versions
    keep = set(os.path.basename(o) for o in objs + mains)
    for f in os.listdir(OBJ):
        if f not in keep:
            os.unlink(os.path.join(OBJ, f))
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", "--jobs", type=int, default=0)
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.jobs, a.verbose, a.force))


if __name__ == "__main__":
    sys.exit(main())
