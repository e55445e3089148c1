"""The drop-in, proven with the reference's own code: the reference's GPU
executables (its unmodified sources built with -DEnableCUDA, and with
-DEnableStreams, by oracle/build.py), whose GPU entry points resolve to this
library through include/remc_cudaexterns.h, run on the B200:

  * its -c check (simulation engine/src/main.cpp:1652-1707): Replica::E() on
    the CPU against Replica::EonDevice() (Replica.cpp:1601-1616, here
    CUDA_EonDevice of libremc_b200.so) on the ten docked reference structures,
    printed as "CPU,GPU,err". The check runs through oracle/ref_gpu_check.cpp,
    the same sequence around the reference's own Replica code with the
    molecule array reserved first: main.cpp's check crashes on the CPU side
    before any GPU work (its stack Replicas delete an uninitialised array
    pointer in Replica::loadMolecule, Replica.cpp:229-245);
  * its start-up check (main.cpp:1745-1797), which warns above 1% relative
    error, followed by a short REMC run whose every Monte Carlo step takes its
    energy from this library (Replica::MCSearch, Replica.cpp:422-426; the
    stream build through CUDA_EonDevice_async and Replica::SumGridResults).

Tolerance: the GPU energy within 1e-5 relative of the reference's own CPU
energy (1e-6 kcal/mol absolute for the one structure near zero).
"""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = {b: os.path.join(ROOT, "oracle", "_ref", b)
       for b in ("REMCDockingGPU", "REMCDockingGPU_streams", "ref_gpu_check")}
E_RTOL = 1e-5


def _need(build):
    if not os.path.exists(EXE[build]):
        pytest.skip("the reference's GPU build is not present (built where the reference is)")


def _write_inputs(d, golden, table):
    """data/AminoAcids, data/pair_potentials_MJ1996 and data/conf{1..10}/1{a,b}.pdb
    (the ten docked reference structures, one chain per file, as the -c
    check reads them)."""
    from remcdockingsimulator_b200.model import write_pdb_ca
    os.makedirs(os.path.join(d, "data"), exist_ok=True)
    table.write(os.path.join(d, "data", "AminoAcids"))
    table.write_pairs(os.path.join(d, "data", "pair_potentials_MJ1996"))
    for k, st in enumerate(golden["structures"]):
        cd = os.path.join(d, "data", "conf%d" % (k + 1))
        os.makedirs(cd, exist_ok=True)
        for c, name in zip(st["chains"], ("1a.pdb", "1b.pdb")):
            write_pdb_ca(os.path.join(cd, name), c["types"], np.array(c["pos"], np.float32),
                         table, chain="A")


def _run(build, args, cwd, timeout=600):
    r = subprocess.run([EXE[build]] + args, cwd=cwd, capture_output=True, text=True,
                       timeout=timeout)
    assert r.returncode == 0, (r.returncode, r.stdout[-3000:], r.stderr[-3000:])
    return r.stdout


def test_reference_check_mode_through_this_library(golden, golden_table, tmp_path, built_lib):
    _need("ref_gpu_check")
    d = str(tmp_path)
    _write_inputs(d, golden, golden_table)
    out = _run("ref_gpu_check", [], d)
    rows = [tuple(float(x) for x in m.groups())
            for m in re.finditer(r"CPU,GPU,err:\s+(\S+)\s+(\S+)\s+(\S+)", out)]
    assert len(rows) == 10, out[-3000:]
    for k, (cpu, gpu, err) in enumerate(rows):
        ref = golden["structures"][k]["reference_E"]
        # the reference's CPU energy here is the reference's E() in the pins
        assert abs(cpu - ref) <= 1e-6 * max(abs(ref), 1.0), (k, cpu, ref)
        if abs(cpu) > 1e-2:
            assert abs(gpu - cpu) <= E_RTOL * abs(cpu), (k, cpu, gpu)
        else:
            assert abs(gpu - cpu) <= 1e-6, (k, cpu, gpu)


@pytest.mark.parametrize("build", ["REMCDockingGPU", "REMCDockingGPU_streams"])
def test_reference_startup_check_and_run_through_this_library(build, golden, golden_table,
                                                              tmp_path, built_lib):
    _need(build)
    d = str(tmp_path)
    _write_inputs(d, golden, golden_table)
    threads = 2
    cfg = os.path.join(d, "config")
    with open(cfg, "w") as fh:
        fh.write("\n".join([
            # sampleafter > 0: the stream build's loop takes the step modulo
            # sampleafter (main.cpp:1042)
            "gpus 1", "streams %d" % threads, "threads %d" % threads, "mcsteps 400",
            "resteps 4", "replicas 4", "samplefrequency 10", "sampleafter 100", "boundry 118.4",
            "temperaturemax 360", "temperaturemin 300", "prefix dropin", "files",
            # structure 3: the chains in contact, E = -10.28 kcal/mol; t(0,0,0)
            # keeps the file's coordinates, angle -1 means no rotation
            "t(0,0,0) r(0,0,1,-1) data/conf3/1a.pdb",
            "t(0,0,0) r(0,0,1,-1) data/conf3/1b.pdb", ""]))
    out = _run(build, ["-f", cfg], d)
    cpu = float(re.search(r"CPU initial energy value:\s+(\S+)", out).group(1))
    gpu = float(re.search(r"GPU initial energy value:\s+(\S+)", out).group(1))
    assert abs(cpu) > 1.0
    assert abs(gpu - cpu) <= E_RTOL * abs(cpu), (cpu, gpu)
    assert "Inconsistency" not in out
    # the REMC run finished and wrote the reference's output files
    files = os.listdir(os.path.join(d, "output"))
    assert any(f.endswith("_fractionBound") for f in files), files
    assert any(f.endswith("_acceptance_ratios") for f in files), files
