"""In-tree build of the CUDA library ``libqgn_b200.so`` (sm_100a) with nvcc.

The library is built next to this file so it travels with the source tree; nothing is
installed into site-packages.  ``python -m qgn_fortran_b200.build`` rebuilds it.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libqgn_b200.so")
OBJDIR = os.path.join(HERE, "_build")
SOURCES = ["rhs_kernels.cu", "layout.cu", "stepper.cu", "capi.cu", "rhs_static.cu", "ensemble.cu", "cnn.cu", "closure.cu",
           "probe.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the QGN CUDA library cannot be built")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    inc = os.path.join(os.path.dirname(HERE), "include")
    hs.extend(os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h"))
    return hs


# the bounds-checked debug build (-DQGN_CHECK): same sources, its own objects and library
CHECK_LIB = os.path.join(HERE, "libqgn_b200_check.so")
CHECK_OBJDIR = os.path.join(HERE, "_build_check")


def build(force: bool = False, verbose: bool = False, check: bool = False) -> str:
    """Build libqgn_b200.so, or with check=True the bounds-checked libqgn_b200_check.so."""
    objdir, lib = (CHECK_OBJDIR, CHECK_LIB) if check else (OBJDIR, LIB)
    extra = ["-DQGN_CHECK"] if check else []
    os.makedirs(objdir, exist_ok=True)
    cc = nvcc()
    headers = _headers()
    jobs = []
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append([cc, *ARCH, *NVCC_FLAGS, *extra, "-c", s, "-o", o])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose and (r.stdout or r.stderr):
            sys.stderr.write(r.stdout + r.stderr)

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    if force or jobs or _stale(lib, objs):
        run([cc, *ARCH, "-shared", "-o", lib, *objs, "-lcudart"])
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, check="--check" in sys.argv))
