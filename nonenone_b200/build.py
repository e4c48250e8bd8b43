"""Build the sm_100a CUDA library in-tree: nonenone_b200/libnonenone_b200.so.

Each per-component-count instantiation is its own translation unit so the
heavy device code compiles in parallel.  Objects go to <repo>/_build/.
Usage: python -m nonenone_b200.build [-v] [--nc 3,4,...]
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
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libnonenone_b200.so")
NC_LIST = (3, 4, 5, 6, 8)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _deps(src: str):
    """A unit depends on its own source and on every header."""
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + [src]
            + [os.path.join(ROOT, "include", "nonenone_b200.h")])


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def units(nc_list=NC_LIST):
    """(source, object, extra flags) for every translation unit."""
    out = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        name = os.path.splitext(os.path.basename(src))[0]
        if name.endswith("_inst") or name == "nz_inst":
            for nc in nc_list:
                out.append((src, os.path.join(BUILD, f"{name}_nc{nc}.o"), [f"-DNZ_INST_NC={nc}"]))
        else:
            out.append((src, os.path.join(BUILD, f"{name}.o"), []))
    return out


def build(verbose: bool = False, nc_list=NC_LIST, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    todo = [u for u in units(nc_list) if _stale(u[1], _deps(u[0]))]
    ptxas = ["-Xptxas", "-v"] if verbose else []

    def compile_one(u):
        src, obj, extra = u
        cmd = [cc, *ARCH, *NVCC_FLAGS, *ptxas, *extra, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {os.path.basename(obj)}:\n{r.stderr[-6000:]}")
        return obj, r.stderr

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            for obj, log in ex.map(compile_one, todo):
                if verbose and log:
                    sys.stderr.write(f"== {os.path.basename(obj)}\n{log}")
    objs = [u[1] for u in units(nc_list)]
    if _stale(LIB, objs):
        cmd = [cc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    return LIB


def build_oracle(verbose: bool = False, reference: str | None = None) -> None:
    """Compile the oracle (test infrastructure): the C restatement always, and
    the reference's own code when the path of its source tree is given
    (`reference`, else the NZ_REFERENCE environment variable) and exists."""
    oracle = os.path.join(ROOT, "oracle")
    targets = ["restatement"]
    ref_root = reference or os.environ.get("NZ_REFERENCE")
    args = []
    if ref_root and os.path.isdir(ref_root):
        targets.append("ref")
        args.append(f"REFERENCE={ref_root}")
    r = subprocess.run(["make", "-C", oracle, *args, *targets],
                       capture_output=not verbose, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{(r.stderr or '')[-4000:]}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--nc", default=",".join(map(str, NC_LIST)))
    ap.add_argument("--oracle", action="store_true")
    ap.add_argument("--reference", default=None,
                    help="source tree of the reference, for the oracle's compiled reference")
    a = ap.parse_args()
    nc_list = tuple(int(x) for x in a.nc.split(","))
    print(build(a.verbose, nc_list))
    if a.oracle:
        build_oracle(a.verbose, a.reference)


if __name__ == "__main__":
    main()
