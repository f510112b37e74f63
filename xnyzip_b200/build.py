"""Builds the in-tree shared library xnyzip_b200/libxnyz.so (and the CLI xnyzip_b200/XnYZip).

CUDA sources are compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
the host sources with the system g++ (the image's $CXX links libstdc++ statically, which
breaks when the library is loaded next to other C++ code).  nvcc cross-compiles without a GPU.

    python xnyzip_b200/build.py            # incremental (not -m: the package needs the library)
    python xnyzip_b200/build.py --force
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libxnyz.so")
CLI = os.path.join(HERE, "XnYZip")
CXX = os.environ.get("XNYZ_CXX", "/usr/bin/g++")
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.path.dirname(os.path.dirname(os.path.realpath(NVCC)))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def find_zstd_157() -> str:
    """Path of the libzstd 1.5.7 shared library bundled on this image ('' if absent)."""
    env = os.environ.get("XNYZ_ZSTD_LIBRARY")
    if env:
        return env
    for root in sorted({sysconfig.get_paths()["purelib"], sysconfig.get_paths()["platlib"]}):
        hits = sorted(glob.glob(os.path.join(root, "pillow.libs", "libzstd-*.so.1.5.7")))
        if hits:
            return hits[0]
    return ""


def _sources():
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "*.cpp")) + glob.glob(os.path.join(CSRC, "host", "*.cpp")))
    return cu, cpp


def _headers():
    return sorted(glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True) +
                  glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True) +
                  glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    cu, cpp = _sources()
    hdrs = _headers()
    zstd = find_zstd_157()
    jobs = []
    objs = []
    for src in cu:
        o = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(o)
        if force or _stale(o, [src] + hdrs):
            jobs.append([NVCC, "-std=c++17", "-O3", "-lineinfo", *ARCH, "-ccbin", CXX, "-Xcompiler", "-fPIC",
                         "-I", CSRC, "-c", src, "-o", o])
    for src in cpp:
        o = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(o)
        if force or _stale(o, [src] + hdrs):
            jobs.append([CXX, "-std=c++17", "-O2", "-fPIC", "-Wall", "-Wextra", "-Wno-unused-parameter",
                         f'-DXNYZ_DEFAULT_ZSTD="{zstd}"', "-I", CSRC, "-I", os.path.join(CUDA_HOME, "include"),
                         "-c", src, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for r in ex.map(_run, jobs):
            if verbose and (r.stdout or r.stderr):
                print(r.stdout, r.stderr, file=sys.stderr)
    if force or jobs or _stale(LIB, objs):
        _run([NVCC, "-shared", *ARCH, "-ccbin", CXX, "-Xcompiler", "-fPIC", "-o", LIB, *objs, "-ldl"])
    cli_src = os.path.join(HERE, "cli", "xnyzip_main.cpp")
    if os.path.exists(cli_src) and (force or _stale(CLI, [cli_src, LIB] + hdrs)):
        _run([CXX, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), cli_src, "-o", CLI,
              "-L", HERE, "-lxnyz", f"-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
