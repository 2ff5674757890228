"""Build libgmg_b200.so (all CUDA kernels + the C ABI) for sm_100a, in-tree.

    python grid-mg-bench_b200/build.py [--verbose-ptxas] [--force]

Objects go to grid-mg-bench_b200/_build/, the library to
grid-mg-bench_b200/libgmg_b200.so (next to this file).  Rebuilds only what
changed (source or shared header newer than its object).
"""
import argparse
import concurrent.futures
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgmg_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xcompiler", "-Wno-unused-parameter"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h")) +
            glob.glob(os.path.join(INCLUDE, "*.hpp")))


def _stale(src, obj, hdr_mtime):
    if not os.path.exists(obj):
        return True
    m = os.path.getmtime(obj)
    return os.path.getmtime(src) > m or hdr_mtime > m


def build(force=False, verbose_ptxas=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [0])
    cc = nvcc()
    todo = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(s, o, hdr_mtime):
            cmd = [cc] + ARCH + FLAGS + ["-I", INCLUDE, "-c", s, "-o", o]
            if verbose_ptxas:
                cmd += ["-Xptxas", "-v"]
            todo.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    failed = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for cmd, r in ex.map(run, todo):
            if r.returncode != 0 or verbose_ptxas:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                failed.append(cmd[-3])
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    relinked = False
    if todo or not os.path.exists(LIB) or force:
        cmd = [cc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcuda"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
        relinked = True
    # host programs over the C++ surface (include/gmg.hpp), linked against the library
    for src in sorted(glob.glob(os.path.join(HERE, "host", "*.cpp"))):
        exe = os.path.join(BUILD, os.path.basename(src)[:-4])
        if force or relinked or _stale(src, exe, hdr_mtime):
            cmd = [cc, "-O2", "-std=c++17", "-I", INCLUDE, src, "-o", exe, "-L", HERE, "-lgmg_b200",
                   "-Xlinker", "-rpath=$ORIGIN/..", "-lcudart"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"host program {src} failed to build:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose_ptxas=a.verbose_ptxas))
