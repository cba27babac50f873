"""Build libephmc_cuda.so in-tree with nvcc for sm_100a.

    python electron-phonon-hmc_b200/build.py            # build if sources changed
    python electron-phonon-hmc_b200/build.py --force    # rebuild

The library is a plain C-ABI shared object (no torch types); the Python
package (``ephmc``) loads it with ctypes.  Output:
``electron-phonon-hmc_b200/lib/libephmc_cuda.so``.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libephmc_cuda.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
           "--expt-relaxed-constexpr"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h")))


def stale():
    if not os.path.exists(LIB) or not all(os.path.exists(os.path.join(LIBDIR, p)) for p in PROGRAMS):
        return True
    t = os.path.getmtime(LIB)
    progs = [os.path.join(CSRC, s) for s in PROGRAMS.values()]
    return any(os.path.getmtime(f) > t for f in sources() + headers() + progs + [__file__])


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc(), *ARCH, *NVFLAGS, "-I", INCLUDE, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode(errors="replace")))
        elif verbose and out:
            print(out.decode(errors="replace"))
    if failed:
        msg = "\n".join(f"--- {s}\n{o}" for s, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-lcusolver", "-lcublas"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    build_programs(verbose)
    return LIB


PROGRAMS = {"organic_conv": "organic_conv_main.cpp"}


def build_programs(verbose=False):
    """Command-line programs over the library (the reference's organic_conv
    interface), linked with an rpath to the library's directory."""
    for name, src in PROGRAMS.items():
        out = os.path.join(LIBDIR, name)
        cmd = ["g++", "-O2", "-std=c++17", "-I", INCLUDE, os.path.join(CSRC, src), "-o", out, "-L", LIBDIR,
               "-lephmc_cuda", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
    sys.exit(0)
