"""Builds the in-tree shared library mpi_3dcompact_b200/libmc3d.so (sm_100a).

    python -m mpi_3dcompact_b200.build [--jobs N] [--force]

Every .cu/.cpp file under csrc/ is compiled with nvcc for sm_100a only and
linked into one shared object exporting the C ABI of include/mc3d.h.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import hashlib
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmc3d.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _digest(extra=()) -> str:
    h = hashlib.sha256()
    for p in _sources() + sorted(glob.glob(os.path.join(CSRC, "*.h"))) + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) \
            + [os.path.join(ROOT, "include", "mc3d.h")]:
        with open(p, "rb") as f:
            h.update(p.encode() + f.read())
    h.update(" ".join(ARCH + FLAGS + list(extra)).encode())
    return h.hexdigest()


def build(force: bool = False, jobs: int = 0, verbose: bool = False) -> str:
    stamp = LIB + ".stamp"
    dig = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp) and open(stamp).read() == dig:
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    cc = nvcc()
    srcs = _sources()

    def comp(src):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        cmd = [cc, *ARCH, *FLAGS, "-c", src, "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stderr}")
        return obj, r.stderr

    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(comp, srcs))
    if verbose:
        for _, err in results:
            if err:
                sys.stderr.write(err)
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    r = subprocess.run([cc, *ARCH, "-shared", "-o", tmp, *objs, "-lcuda"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stderr)
    os.replace(tmp, LIB)
    with open(stamp, "w") as f:
        f.write(dig)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose))
