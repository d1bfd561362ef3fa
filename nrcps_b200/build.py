"""Builds libnrcps_b200.so in-tree (nrcps_b200/libnrcps_b200.so) for sm_100a.

    python -m nrcps_b200.build [--jobs N] [--force]

Every .cu under csrc/ is compiled with nvcc for compute_100a/sm_100a (the
B200's architecture-specific target); host-only .cc files with g++; the
objects are linked into one shared library whose exported symbols are the
C ABI of include/nrcps_b200.h.  Objects go to nrcps_b200/_build/ (git-ignored).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnrcps_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I", os.path.join(REPO, "include")] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-I", os.path.join(REPO, "include")]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu"))), sorted(glob.glob(os.path.join(CSRC, "*.cc")))


def _obj(src: str) -> str:
    return os.path.join(OBJ, os.path.basename(src) + ".o")


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(REPO, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _stale(src: str, obj: str, hdr: float) -> bool:
    return not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr)


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    return cmd, r.returncode, r.stdout + r.stderr


def build(jobs: int = 8, force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    cus, ccs = _sources()
    hdr = _headers_mtime()
    cmds = []
    for s in cus:
        o = _obj(s)
        if force or _stale(s, o, hdr):
            cmds.append([NVCC, *NVCC_FLAGS, "-c", s, "-o", o])
    for s in ccs:
        o = _obj(s)
        if force or _stale(s, o, hdr):
            cmds.append(["g++", *CXX_FLAGS, "-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        for cmd, rc, out in ex.map(_compile, cmds):
            if verbose or rc != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + out)
            if rc != 0:
                raise RuntimeError(f"compilation failed: {os.path.basename(cmd[-3])}")
    objs = [_obj(s) for s in cus + ccs]
    if force or cmds or not os.path.exists(LIB):
        link = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(link, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(" ".join(link) + "\n" + r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 8)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.jobs, a.force, a.verbose))
