"""Builds the library in-tree: graph_analytics_applesilicon_b200/libgraphb200.so
(every .cu / .cpp under csrc/, compiled by nvcc for sm_100a) and the command-line
programs bin/gbench (benchmark + validation) and bin/gconvert (SNAP -> .bin).

    python -m graph_analytics_applesilicon_b200.build [--force] [--verbose]

Objects go to _build/ and are rebuilt when a source or any header is newer.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libgraphb200.so")
GBENCH = os.path.join(PKG, "bin", "gbench")
PROGRAMS = ("gbench", "gconvert")  # csrc/<name>.cpp -> bin/<name>
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-fopenmp",
              "-I" + os.path.join(ROOT, "include"), "-I" + CSRC] + ARCH


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "*.h*")) + glob.glob(os.path.join(CSRC, "*.cuh"))
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, force: bool, verbose: bool, extra: list[str]) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and not _stale(obj, [src] + _headers()):
        return obj
    cmd = [nvcc(), "-c", src, "-o", obj] + NVCC_FLAGS + extra
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, flush=True)
    return obj


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(GBENCH), exist_ok=True)
    lib_srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    lib_srcs = [s for s in lib_srcs if os.path.splitext(os.path.basename(s))[0] not in PROGRAMS]
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force or ptxas_info, verbose or ptxas_info, extra), lib_srcs))
    if force or _stale(LIB, objs):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-Xcompiler", "-fopenmp", "-lgomp", "-lz"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    for prog in PROGRAMS:
        src, exe = os.path.join(CSRC, prog + ".cpp"), os.path.join(PKG, "bin", prog)
        if os.path.exists(src) and (force or _stale(exe, [src, LIB] + _headers())):
            cmd = ["g++", "-std=c++17", "-O2", "-fopenmp", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, src,
                   "-o", exe, "-L" + PKG, "-lgraphb200", "-Wl,-rpath,$ORIGIN/.."]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"{prog} build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="rebuild with -Xptxas -v")
    a = ap.parse_args()
    try:
        print(build(a.force, a.verbose, a.ptxas_info))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
