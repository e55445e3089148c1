"""Build the engine's CUDA shared library in-tree for sm_100a.

  python -m remcdockingsimulator_b200.build [--force]

Produces remcdockingsimulator_b200/lib/libremc_b200.so from csrc/*.cu with
nvcc (-gencode arch=compute_100a,code=sm_100a). The library exports the C ABI
declared in include/remc_b200.h and include/remc_reference_abi.h. Then builds
the C++ Replica/Molecule facade over it (csrc/remc_replica.{h,cpp}) into
lib/libremc_replica.so and its command-line check driver lib/remc_replica_check.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libremc_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


FACADE = os.path.join(LIBDIR, "libremc_replica.so")
FACADE_CHECK = os.path.join(LIBDIR, "remc_replica_check")
CXX = os.environ.get("CXX", "g++")
# no FMA contraction: host move arithmetic rounds like the reference's
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall",
            "-I" + os.path.join(ROOT, "include")]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps() -> list[str]:
    hdrs = [h for h in glob.glob(os.path.join(CSRC, "*.h"))
            if not os.path.basename(h).startswith("remc_replica")]
    return (sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + hdrs
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in _deps())


def _facade_stale() -> bool:
    deps = [LIB] + glob.glob(os.path.join(CSRC, "remc_replica*")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    outs = [FACADE, FACADE_CHECK]
    if not all(os.path.exists(o) for o in outs):
        return True
    t = min(os.path.getmtime(o) for o in outs)
    return any(os.path.getmtime(d) > t for d in deps)


def build_facade(force: bool = False) -> str:
    """g++ build of the C++ facade, linked against libremc_b200.so."""
    if not force and not _facade_stale():
        return FACADE
    rpath = "-Wl,-rpath,$ORIGIN"
    steps = [
        [CXX] + CXXFLAGS + ["-shared", os.path.join(CSRC, "remc_replica.cpp"), "-o",
                            FACADE + ".tmp", "-L" + LIBDIR, "-lremc_b200", rpath],
    ]
    for cmd in steps:
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("facade build failed:\n%s%s" % (r.stdout, r.stderr))
    os.replace(FACADE + ".tmp", FACADE)
    cmd = [CXX] + CXXFLAGS + [os.path.join(CSRC, "remc_replica_check.cpp"), "-o",
                              FACADE_CHECK + ".tmp", "-L" + LIBDIR, "-lremc_replica",
                              "-lremc_b200", rpath]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("facade check build failed:\n%s%s" % (r.stdout, r.stderr))
    os.replace(FACADE_CHECK + ".tmp", FACADE_CHECK)
    return FACADE


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        build_facade(force)
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    build_facade(force=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
