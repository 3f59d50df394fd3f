"""Build ``pict_b200/libpict_b200.so`` (the C-ABI library) with nvcc for sm_100a.

The library is built in-tree so the shared object travels with the source tree.
Every ``.cu``/``.cpp`` file in ``pict_b200/csrc`` is compiled to an object
file under ``pict_b200/_build`` (in parallel) and linked into one shared
library; recompilation is skipped when no source or header is newer than the
library.

Usage::

    python -m pict_b200.build [--force] [--verbose] [--ptxas-info]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpict_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = os.path.join(cuda, "bin", "nvcc")
    if os.path.exists(p):
        return p
    p = shutil.which("nvcc")
    if p is None:
        raise RuntimeError("nvcc not found")
    return p


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _deps():
    return _sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h")) + [os.path.abspath(__file__)]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in _deps())


def _compile(src, extra, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    cmd = [_nvcc(), "-c", src, "-o", obj, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
           "-I", INCLUDE, "-I", CSRC] + ARCH + extra
    if src.endswith(".cpp"):
        cmd = [_nvcc(), "-c", src, "-o", obj, "-std=c++17", "-O3", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    return obj, r.stderr


def build(force=False, verbose=False, ptxas_info=False):
    if not force and not needs_build():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, extra, verbose), srcs))
    if ptxas_info:
        for _, err in results:
            sys.stderr.write(err)
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), "-shared", "-o", tmp] + objs + ARCH + ["-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force or a.ptxas_info, verbose=a.verbose, ptxas_info=a.ptxas_info))


if __name__ == "__main__":
    main()
