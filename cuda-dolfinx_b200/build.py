"""Build libcudolfinx_b200.so (sm_100a) in-tree.

    python cuda-dolfinx_b200/build.py [--verbose-ptxas] [--force]

Steps: regenerate csrc/fe_element_code.cuh from csrc/gen_element_code.py,
compile every csrc/*.cu with nvcc for sm_100a and csrc/*.cpp with g++, link
lib/libcudolfinx_b200.so.  Objects go to _build/ (git-ignored); rebuilds are
incremental on source/header modification times.
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
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libcudolfinx_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newer(dst, srcs):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(s) > t for s in srcs)


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
            + [os.path.join(ROOT, "include", "cudolfinx_b200.h")])


def _compile(src, verbose_ptxas):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not _newer(obj, [src] + _headers()):
        return obj, ""
    if src.endswith(".cu"):
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
               "-Xcompiler", "-fPIC", "-c", src, "-o", obj]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
    else:
        cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-pthread", "-I/usr/local/cuda/include", "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force=False, verbose_ptxas=False, quiet=True):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_element_code.py")])
    if force:
        for o in glob.glob(os.path.join(BUILD, "*.o")):
            os.remove(o)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    objs = [o for o, _ in results]
    for _, log in results:
        if log and (verbose_ptxas or not quiet):
            print(log)
    if _newer(LIB, objs):
        tmp = LIB + f".tmp{os.getpid()}"
        # NVRTC compiles forms given as FFCx tabulate_tensor bodies at run time
        cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lpthread", "-lnvrtc"]
        subprocess.check_call(cmd)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose_ptxas=a.verbose_ptxas, quiet=False))
