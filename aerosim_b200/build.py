"""Builds libaerosim.so (sm_100a) in-tree with nvcc.

Usage: python -m aerosim_b200.build [--force]

Translation units and their floating-point contracts:
  lbm_fast.cu   storage-type dispatch of the FP32-arithmetic step kernels
  lbm_fast_<s>.cu  FP32-arithmetic step kernels per storage type, FMA contraction allowed
  lbm_exact.cu  FP64 kernels mirroring the reference's rounding: -fmad=false
  voxelize.cu   FP64 BVH voxelizer, bit-exact flags and links: -fmad=false
  engine.cu     C-ABI host layer
  noalloc.cu    allocation-free force reduction entry point: -fmad=false
  sgs.cu        learned SGS closure: MLP training, wall distance, training samples
  mesh.cu       STL reader, mesh statistics, frontal-area raster kernel: -fmad=false
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libaerosim.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
          "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", CSRC, "-I", INCLUDE]
UNITS = {
    "lbm_fast.cu": [],
    "lbm_fast_f32.cu": [],
    "lbm_fast_f16s.cu": [],
    "lbm_fast_bf16s.cu": [],
    "lbm_fast_f16c.cu": [],
    "lbm_exact.cu": ["-fmad=false"],
    "voxelize.cu": ["-fmad=false"],
    "engine.cu": [],
    "noalloc.cu": ["-fmad=false"],
    "sgs.cu": [],
    "mesh.cu": ["-fmad=false"],
}


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libaerosim.so")
    return exe


def _deps() -> list[str]:
    out = []
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h")):
                out.append(os.path.join(d, f))
    return out


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compiles every translation unit for sm_100a and links libaerosim.so."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    deps = _deps()
    exe = nvcc()
    jobs = []
    for unit, flags in UNITS.items():
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        if force or _stale(obj, deps):
            cmd = [exe, *ARCH, *COMMON, *flags]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            cmd += ["-c", os.path.join(CSRC, unit), "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for msg in ex.map(run, jobs):
            if ptxas_info and msg:
                print(msg)
    objs = [os.path.join(BUILD, u.replace(".cu", ".o")) for u in UNITS]
    if force or jobs or _stale(LIB, objs):
        cmd = [exe, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static"]
        run(cmd)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_info=a.ptxas_info))
    sys.exit(0)
