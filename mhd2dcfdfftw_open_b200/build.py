"""Build the sm_100a shared library in-tree.

``python -m mhd2dcfdfftw_open_b200.build`` compiles every ``csrc/*.cu`` with
nvcc for sm_100a (``-gencode arch=compute_100a,code=sm_100a``) into
``mhd2dcfdfftw_open_b200/libmhdgpu.so`` and the drop-in object
``csrc/dropin.c`` into ``libmhdgpu_dropin.a``.  No GPU is needed to build.
"""
from __future__ import annotations

import concurrent.futures
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libmhdgpu.so")
DROPIN = os.path.join(PKG, "libmhdgpu_dropin.a")
BUILD_DIR = os.path.join(ROOT, "_build")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD_DIR, exist_ok=True)
    cus = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdrs = sorted(glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(ROOT, "include", "*.h")))
    objs, cmds = [], []
    for cu in cus:
        obj = os.path.join(BUILD_DIR, os.path.basename(cu) + ".o")
        objs.append(obj)
        if force or _stale(obj, [cu] + hdrs):
            cmds.append([nvcc()] + NVCC_FLAGS + ["-dc", cu, "-o", obj])
    # the translation units are independent: compile them side by side
    with concurrent.futures.ThreadPoolExecutor(max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd))
        for f in [ex.submit(subprocess.run, cmd, check=True) for cmd in cmds]:
            f.result()
    if force or _stale(LIB, objs):
        cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
               "-Xcompiler", "-fPIC", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    dropin_c = os.path.join(CSRC, "dropin.c")
    if os.path.exists(dropin_c) and (force or _stale(DROPIN, [dropin_c] + hdrs)):
        obj = os.path.join(BUILD_DIR, "dropin.o")
        subprocess.run(["gcc", "-O2", "-fPIC", "-std=c99", "-c", dropin_c,
                        "-I", os.path.join(ROOT, "include"), "-o", obj], check=True)
        if os.path.exists(DROPIN):
            os.remove(DROPIN)
        subprocess.run(["ar", "rcs", DROPIN, obj], check=True)
    return LIB


def build_dropin_demo(ref_dir: str | None = None) -> None:
    """Link the reference's own driver against the drop-in layer (needs the
    reference sources: `ref_dir`, else $MHD_REF_DIR, else the default of
    oracle/Makefile; outputs go to oracle/_ref/)."""
    build()
    d = ref_dir or os.environ.get("MHD_REF_DIR")
    cmd = ["make", "-s", "-C", os.path.join(ROOT, "oracle")] + ([f"REF_DIR={d}"] if d else [])
    subprocess.run(cmd + ["dropin"], check=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
