"""Builds libsfac.so (the C-ABI library with the sm_100a kernels) in-tree.

    python -m ewaldcorrel_b200.build [--force] [--verbose] [--check]

nvcc cross-compiles for sm_100a without a GPU.  Objects go to
ewaldcorrel_b200/_build/, the shared library to ewaldcorrel_b200/libsfac.so
(next to ewald.py, which loads it from its own directory like the
reference's wrapper does, ewald.py:52-53).

--check builds the index-checking variant instead (-DSPME_CHECK: kernels
test their indices and record the first failure in an error word rather
than trapping): objects in _build_check/, library libsfac_check.so, loaded
by ewald.py when EWALDCORREL_LIBSFAC names it.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libsfac.so")
BUILD_CHECK = os.path.join(PKG, "_build_check")
LIB_CHECK = os.path.join(PKG, "libsfac_check.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC,-O3,-ffp-contract=off,-fno-strict-aliasing",
    "-Xptxas",
    "-warn-spills",
]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if os.path.exists(cand) else "nvcc"


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else -1.0


def build(force: bool = False, verbose: bool = False, check: bool = False) -> str:
    """Compiles every .cu under csrc/ for sm_100a and links libsfac.so
    (libsfac_check.so with -DSPME_CHECK when check is set)."""
    bdir, lib = (BUILD_CHECK, LIB_CHECK) if check else (BUILD, LIB)
    extra = ["-DSPME_CHECK"] if check else []
    os.makedirs(bdir, exist_ok=True)
    nvcc = _nvcc()
    hdr_time = max([_mtime(h) for h in _headers()] + [_mtime(__file__)])
    jobs = []
    objs = []
    for src in _sources():
        obj = os.path.join(bdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _mtime(obj) < max(_mtime(src), hdr_time):
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, *extra, "-I", CSRC, "-I", INCLUDE, "-c", src, "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, flush=True)
        return r

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    if jobs or force or _mtime(lib) < max(_mtime(o) for o in objs):
        cmd = [nvcc, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", lib, *objs]
        run(cmd)
    return lib


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--check", action="store_true", help="index-checking build (libsfac_check.so)")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose, check=a.check))


if __name__ == "__main__":
    sys.exit(main())
