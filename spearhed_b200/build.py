"""Builds the CUDA library in-tree: spearhed_b200/_lib/libspearhed_b200.so,
and its bounds-checked twin spearhed_b200/_lib/libspearhed_b200_check.so
(compiled with -DSPH_CHECK: device index checks that report a failed check in
a status word and skip the access; loaded when SPEARHED_B200_VARIANT=check).

Every translation unit is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``); there is no other target.
Objects are rebuilt when their source or any header in csrc/ or include/ is newer.

    python -m spearhed_b200.build [--verbose] [--ptxas-info] [--no-check]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT, "libspearhed_b200.so")
CHECK_OUT = os.path.join(OUT, "check")
CHECK_LIB = os.path.join(OUT, "libspearhed_b200_check.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I", os.path.join(ROOT, "include")]


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src, obj, extra, verbose):
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return r.stderr


def _build_variant(out, lib, defines, verbose, ptxas_info, force):
    os.makedirs(out, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr = _newest_header()
    jobs = []
    for s in srcs:
        obj = os.path.join(out, os.path.basename(s)[:-3] + ".o")
        if force or ptxas_info or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(s), hdr):
            jobs.append((s, obj))
    extra = defines + (["-Xptxas", "-v"] if ptxas_info else [])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            futs = {ex.submit(_compile, s, o, extra, verbose): s for s, o in jobs}
            for f in cf.as_completed(futs):
                err = f.result()
                if ptxas_info and err:
                    print(f"== {os.path.basename(futs[f])}\n{err}")
    objs = [os.path.join(out, os.path.basename(s)[:-3] + ".o") for s in srcs]
    if jobs or not os.path.exists(lib):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return lib


def build(verbose=False, ptxas_info=False, force=False, check=True):
    """Builds the library, and (check=True) its bounds-checked twin."""
    _build_variant(OUT, LIB, [], verbose, ptxas_info, force)
    if check and not ptxas_info:
        _build_variant(CHECK_OUT, CHECK_LIB, ["-DSPH_CHECK"], verbose, False, force)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--no-check", action="store_true", help="skip the bounds-checked twin")
    a = ap.parse_args()
    print(build(verbose=a.verbose, ptxas_info=a.ptxas_info, force=a.force, check=not a.no_check))
    sys.exit(0)
