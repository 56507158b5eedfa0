"""Builds the CUDA libraries in-tree: ns3dperiodic_b200/libns3d_b200.so (the
C ABI of include/ns3d.h) and ns3dperiodic_b200/libns3d_compat.so (the
reference-signature C++ layer of include/ns3d_compat.h over that ABI).

nvcc for sm_100a only, one object per translation unit (compiled in
parallel).  Usage: ``python -m ns3dperiodic_b200.build [-j N]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(HERE, "libns3d_b200.so")
COMPAT_LIB = os.path.join(HERE, "libns3d_compat.so")
COMPAT_SOURCE = "compat.cu"

SOURCES = ["k_fwdx.cu", "k_fwdx32.cu", "k_xy.cu", "k_xy_rev.cu", "k_z.cu", "k_fft3d.cu", "aux_kernels.cu", "solver.cu",
           "noalloc.cu", "krylov.cu", "qr_shifts.cpp", "checkpoint.cpp",
           "diag_kernels.cu", "series.cpp", "server.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-Xptxas", "-v", "-I" + os.path.join(ROOT, "include")] + ARCH


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _compile(src: str) -> tuple[str, str]:
    out = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    cmd = [nvcc(), *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
    return out, r.stderr


def _stale(objs) -> bool:
    if not os.path.exists(LIB) or not os.path.exists(COMPAT_LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    return any(os.path.getmtime(d) > t for d in deps)


def build(jobs: int = 0, force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    if not force and not _stale(None):
        return LIB
    jobs = jobs or min(len(SOURCES), os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(_compile, SOURCES))
    log = os.path.join(ROOT, "_build", "ptxas.log")
    with open(log, "w") as f:
        for _, err in results:
            f.write(err)
    objs = [o for o, _ in results]
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    # the reference-signature C++ layer over the C ABI, in its own library
    cobj, _ = _compile(COMPAT_SOURCE)
    cmd = [nvcc(), *ARCH, "-shared", "-o", COMPAT_LIB, cobj, "-L" + HERE, "-lns3d_b200",
           "-Xlinker", "-rpath=$ORIGIN", "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compat link failed:\n{r.stderr}")
    if verbose:
        print("built", LIB, file=sys.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=0)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.force, verbose=True))
