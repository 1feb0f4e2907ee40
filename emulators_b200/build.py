"""Build the sm_100a shared library ``emulators_b200/libemusv_b200.so`` with nvcc.

The library is compiled in-tree so it travels with the repository snapshot; there is
no JIT step at import time.  Usage: ``python -m emulators_b200.build [--force] [-v]``.
"""

from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(REPO, "include")
OBJDIR = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libemusv_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
         "-I", INCLUDE, "-I", CSRC]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps() -> list[str]:
    return (sources() + glob.glob(os.path.join(CSRC, "*.cuh"))
            + glob.glob(os.path.join(INCLUDE, "*.h")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    jobs = []
    for src in sources():
        obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")
        jobs.append(([NVCC, *ARCH, *FLAGS, *extra, "-c", src, "-o", obj], obj))
    if verbose:
        for cmd, _ in jobs:
            print(" ".join(cmd), flush=True)
    # one nvcc per translation unit, run side by side (ptxas output stays per file)
    workers = max(1, min(len(jobs), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        results = list(ex.map(lambda j: subprocess.run(j[0], capture_output=True, text=True), jobs))
    for (cmd, _), r in zip(jobs, results):
        if r.stdout or r.stderr:
            sys.stdout.write(r.stdout + r.stderr)
        if r.returncode:
            raise subprocess.CalledProcessError(r.returncode, cmd)
    objs = [obj for _, obj in jobs]
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register/smem usage")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas))
    return 0


if __name__ == "__main__":
    sys.exit(main())
