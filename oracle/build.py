"""Build recipe for the test oracles (TEST INFRASTRUCTURE).

Produces:
  oracle/_build/libremc_oracle.so  - the FP64 C restatement (remc_oracle.c)
  oracle/_ref/libremcref.so        - the reference CPU engine's own sources
                                     (compiled unmodified from the reference
                                     tree) + ref_harness.cpp
  oracle/_ref/REMCDockingCPU       - the reference CPU executable, same sources
                                     + its main.cpp
  oracle/_ref/REMCDockingGPU       - the reference's own GPU build (-DEnableCUDA),
  oracle/_ref/REMCDockingGPU_streams  and its stream build (-DEnableStreams),
  oracle/_ref/ref_gpu_check          the -c check of the GPU build's main.cpp
                                     around its own Replica code (ref_gpu_check.cpp),
                                     from the same unmodified sources, with
                                     include/remc_cudaexterns.h force-included
                                     in place of its cudaExterns.h and linked
                                     against this repository's libremc_b200.so
                                     instead of its CudaFunctions.cu

The reference tree is read where it lies: the directory REMC_REFERENCE_ROOT
names, by default a directory `reference` beside this repository's root, and
its `simulation engine/src`; nothing is copied into this repository. Missing GSL / cutil headers are
replaced by the project-written stubs in oracle/ref_stubs/. When the tree is
absent (e.g. on a machine that only received the prebuilt files) the
reference build is skipped and the prebuilt files are used as they are.

Usage: python oracle/build.py [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
STUBS = os.path.join(HERE, "ref_stubs")
REF_UNITS = ["AminoAcid", "AminoAcids", "Link", "Molecule", "Quaternion", "Replica", "Residue",
             "TorsionalLookupMatrix", "vector3f"]
# the reference's own CPU flags (simulation engine/Makefile:17); gnu++11 only
# because the stubs use <chrono>; -fpermissive for its pre-standard C++.
REF_CFLAGS = ["-std=gnu++11", "-fpermissive", "-w", "-O2", "-fno-omit-frame-pointer", "-fPIC",
              "-pthread"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "remc_oracle.c")
    out = os.path.join(BUILD, "libremc_oracle.so")
    if force or _stale(out, [src, os.path.join(HERE, "remc_oracle.h")]):
        # default x86-64 target: no FMA, so FP32/FP64 ops round like the reference's
        _run(["gcc", "-O2", "-fPIC", "-shared", "-std=c99", "-o", out, src, "-lm"])
    return out


def reference_root() -> str:
    """Root of the reference project: $REMC_REFERENCE_ROOT, else `reference`
    beside this repository's root."""
    repo = os.path.dirname(HERE)
    return os.environ.get("REMC_REFERENCE_ROOT",
                          os.path.join(os.path.dirname(repo), "reference"))


def reference_src() -> str:
    return os.path.join(reference_root(), "simulation engine", "src")


def build_reference(force: bool = False) -> bool:
    """Compile the reference engine (unmodified) + harness. Returns False when
    the reference tree is not present here."""
    src_dir = reference_src()
    if not os.path.isdir(src_dir):
        return False
    os.makedirs(REF_OUT, exist_ok=True)
    objdir = os.path.join(REF_OUT, "obj")
    os.makedirs(objdir, exist_ok=True)
    inc = ["-I" + STUBS, "-I" + src_dir, "-I/usr/local/cuda/include"]
    stub_files = [os.path.join(dp, f) for dp, _, fs in os.walk(STUBS) for f in fs]
    objs = []
    for unit in REF_UNITS + ["main"]:
        s = os.path.join(src_dir, unit + ".cpp")
        o = os.path.join(objdir, unit + ".o")
        if force or _stale(o, [s] + stub_files):
            _run(["g++"] + REF_CFLAGS + inc + ["-c", s, "-o", o])
        objs.append(o)
    harness_src = os.path.join(HERE, "ref_harness.cpp")
    harness_obj = os.path.join(objdir, "ref_harness.o")
    if force or _stale(harness_obj, [harness_src] + stub_files):
        _run(["g++"] + REF_CFLAGS + inc + ["-c", harness_src, "-o", harness_obj])
    lib = os.path.join(REF_OUT, "libremcref.so")
    lib_objs = [o for o in objs if not o.endswith("main.o")] + [harness_obj]
    if force or _stale(lib, lib_objs):
        _run(["g++", "-shared", "-pthread", "-o", lib] + lib_objs + ["-lpthread"])
    exe = os.path.join(REF_OUT, "REMCDockingCPU")
    main_objs = [o for o in objs]
    if force or _stale(exe, main_objs):
        # -lcudart only for the one cudaGetErrorString call (main.cpp:1281)
        _run(["g++", "-o", exe] + main_objs +
             ["-lpthread", "-L/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath,/usr/local/cuda/lib64"])
    return True


def build_reference_gpu(force: bool = False) -> bool:
    """The reference's own GPU executables, linked against libremc_b200.so:
    every unit of the reference compiled unmodified with -DEnableCUDA (and
    -DEnableStreams for the stream build), with include/remc_cudaexterns.h
    force-included so that its `#include "cudaExterns.h"` resolves to this
    library's entry points. Needs the engine library built first. Returns
    False when the reference tree or the library is absent."""
    src_dir = reference_src()
    repo = os.path.dirname(HERE)
    libdir = os.path.join(repo, "remcdockingsimulator_b200", "lib")
    lib = os.path.join(libdir, "libremc_b200.so")
    if not os.path.isdir(src_dir) or not os.path.exists(lib):
        return False
    shim = os.path.join(repo, "include", "remc_cudaexterns.h")
    inc = ["-I" + STUBS, "-I" + src_dir, "-I" + os.path.join(repo, "include"),
           "-I/usr/local/cuda/include", "-include", shim]
    deps = ([shim, os.path.join(repo, "include", "remc_reference_abi.h")] +
            [os.path.join(dp, f) for dp, _, fs in os.walk(STUBS) for f in fs])
    for name, defs in (("REMCDockingGPU", ["-DEnableCUDA"]),
                       ("REMCDockingGPU_streams", ["-DEnableCUDA", "-DEnableStreams"])):
        objdir = os.path.join(REF_OUT, "obj_" + name)
        os.makedirs(objdir, exist_ok=True)
        objs = []
        for unit in REF_UNITS + ["main"]:
            s = os.path.join(src_dir, unit + ".cpp")
            o = os.path.join(objdir, unit + ".o")
            if force or _stale(o, [s] + deps):
                _run(["g++"] + REF_CFLAGS + defs + inc + ["-c", s, "-o", o])
            objs.append(o)
        # the library is found next to the repository at run time
        link = ["-pthread", "-L" + libdir, "-lremc_b200", "-L/usr/local/cuda/lib64", "-lcudart",
                "-L/usr/local/cuda/lib64/stubs", "-lcuda",
                "-Wl,-rpath,$ORIGIN/../../remcdockingsimulator_b200/lib",
                "-Wl,-rpath,/usr/local/cuda/lib64"]
        exe = os.path.join(REF_OUT, name)
        if force or _stale(exe, objs + [lib]):
            _run(["g++", "-o", exe] + objs + link)
        if name == "REMCDockingGPU":
            # the -c check around the reference's own Replica code
            chk_src = os.path.join(HERE, "ref_gpu_check.cpp")
            chk_obj = os.path.join(objdir, "ref_gpu_check.o")
            if force or _stale(chk_obj, [chk_src] + deps):
                _run(["g++"] + REF_CFLAGS + defs + inc + ["-c", chk_src, "-o", chk_obj])
            chk = os.path.join(REF_OUT, "ref_gpu_check")
            unit_objs = [o for o in objs if not o.endswith("main.o")]
            if force or _stale(chk, unit_objs + [chk_obj, lib]):
                _run(["g++", "-o", chk] + unit_objs + [chk_obj] + link)
    return True


def main() -> int:
    force = "--force" in sys.argv
    print("oracle:", build_oracle(force))
    print("reference:", "built" if build_reference(force) else "tree absent, skipped")
    print("reference GPU build:",
          "built" if build_reference_gpu(force) else "tree or engine library absent, skipped")
    return 0


if __name__ == "__main__":
    sys.exit(main())
