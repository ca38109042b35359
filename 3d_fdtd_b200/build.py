"""Builds libfdtd_b200.so in-tree (3d_fdtd_b200/lib/) for sm_100a.

    python 3d_fdtd_b200/build.py [--verbose-ptxas] [--force]

Each source in csrc/ is compiled to an object under _build/ (skipped when the
object is newer than every source and header), in parallel, then linked into
one shared library with the CUDA runtime linked statically.  Only nvcc and the
host C++ compiler are needed; no GPU.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build", "fdtd_b200")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libfdtd_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=default",
              "--expt-relaxed-constexpr", "-ccbin", "g++"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _compile(src: str, obj: str, ptxas_v: bool) -> tuple[str, str]:
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", src, "-o", obj]
    if ptxas_v and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{p.stdout}\n{p.stderr}")
    return src, p.stderr


def build(force: bool = False, ptxas_v: bool = False, quiet: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdr_mtime = max((os.path.getmtime(h) for h in _headers()), default=0)
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or ptxas_v or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_mtime):
            jobs.append((s, o))
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for src, log in ex.map(lambda a: _compile(*a, ptxas_v), jobs):
            if log.strip() and (ptxas_v or not quiet):
                print(f"--- {os.path.basename(src)}\n{log}", file=sys.stderr)
    newest = max(os.path.getmtime(o) for o in objs)
    if force or jobs or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static", "-ccbin", "g++"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{p.stdout}\n{p.stderr}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_v=a.verbose_ptxas, quiet=False))


if __name__ == "__main__":
    main()
