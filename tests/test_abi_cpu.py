"""CPU checks of the C ABI: the shared library loads without a GPU and exports
every function declared in include/*.h."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(([^;{}]*)\)\s*;", text):
            name = m.group(1)
            if name in ("if", "while", "for", "return", "sizeof"):
                continue
            names.add(name)
    return names


def test_headers_declare_entry_points():
    names = declared_functions()
    for must in ("remc_create", "remc_sweep", "remc_run", "remc_energy_full", "CUDA_EonDevice",
                 "CUDA_EonDevice_async", "copyLJPotentialDataToDevice", "CUDA_setBoxDimension"):
        assert must in names


def test_library_exports_every_declared_symbol(built_lib):
    lib = ctypes.CDLL(built_lib)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_default_params_are_reference_constants(built_lib):
    import numpy as np
    from remcdockingsimulator_b200._capi import default_params
    from remcdockingsimulator_b200 import model
    p = default_params()
    assert np.float32(p.lambda_) == np.float32(0.159)
    assert np.float32(p.e0) == np.float32(-2.27)
    assert np.float32(p.kbt_cf) == model.KBT_CONVERSION_FACTOR
    assert np.float32(p.dh_const) == model.DH_CONSTANT
    assert np.float32(p.lj_cf) == model.LJ_CONVERSION_FACTOR
    assert p.crowder_mode == 0 and np.float32(p.crowder_cutoff) == np.float32(15.0)
    # the pure-Python copy (used where the engine library must not be loaded,
    # e.g. the benchmark's reference arm) holds the same FP32 values
    from remcdockingsimulator_b200.engine import reference_params
    q = reference_params()
    for name, _ in type(p)._fields_:
        assert getattr(q, name) == getattr(p, name), name


def test_workload_generation_does_not_load_the_engine_library():
    """Building a benchmark workload (what the reference arm of bench.py does)
    maps nothing of this repository's native code."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from remcdockingsimulator_b200 import synth\n"
            "w = synth.two_chain(1)\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libremc_b200' not in maps and 'libremc_replica' not in maps\n"
            "print('clean')\n" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "clean" in r.stdout, r.stderr


def test_create_rejects_bad_descriptors_without_gpu(built_lib):
    """Argument validation happens before any device call."""
    import numpy as np
    from remcdockingsimulator_b200._capi import SystemDesc, lib, default_params, REMC_ERR_INVALID
    ms = np.array([0, 2, 3], np.int32)
    roles = np.array([0, 0], np.int32)
    types = np.array([0, 1, 25], np.int32)  # 25 is not a valid type
    d = SystemDesc()
    d.n_beads, d.n_mol, d.n_replicas = 3, 2, 1
    d.mol_start = ms.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    d.mol_role = roles.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    d.bead_type = types.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    d.box = 50.0
    d.translate_only_crowders = 0
    h = ctypes.c_void_p()
    p = default_params()
    rc = lib().remc_create(ctypes.byref(d), 1, ctypes.byref(p), ctypes.byref(h))
    assert rc == REMC_ERR_INVALID
    assert b"type" in lib().remc_last_error_string()


@pytest.mark.parametrize("exe", ["REMCDockingGPU", "REMCDockingGPU_streams", "ref_gpu_check"])
def test_reference_gpu_build_links_this_library(exe):
    """The reference's own GPU build (its unmodified sources with -DEnableCUDA
    and include/remc_cudaexterns.h force-included, made by oracle/build.py)
    takes its GPU entry points from libremc_b200.so."""
    import subprocess
    path = os.path.join(ROOT, "oracle", "_ref", exe)
    if not os.path.exists(path):
        pytest.skip("the reference's GPU build is made where the reference tree is present")
    out = subprocess.run(["readelf", "-d", path], capture_output=True, text=True).stdout
    assert "libremc_b200.so" in out
    syms = subprocess.run(["nm", "-D", "--undefined-only", path], capture_output=True,
                          text=True).stdout
    for name in ("CUDA_EonDevice", "copyLJPotentialDataToDevice", "CUDA_setBoxDimension"):
        assert name in syms, name
