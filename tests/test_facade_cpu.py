"""CPU checks of the C++ Replica/Molecule facade (csrc/remc_replica.h): its
PDB reader and rigid moves round exactly like the Python model (which follows
Molecule.cpp:88-102, 146-171, 247-346 and Quaternion.cpp:84-101), its table
readers agree with AminoAcidTable, and the library exports the reference's
method names. No call here touches the GPU."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from remcdockingsimulator_b200 import build, synth
from remcdockingsimulator_b200.model import AminoAcidTable, Molecule, normalise_axis


def _check(*args):
    r = subprocess.run([build.FACADE_CHECK] + [str(a) for a in args], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    return r.stdout


def _parse_blocks(out):
    """Blocks of (centre, quat, beads) printed by print_molecule."""
    blocks, cur = [], None
    for ln in out.splitlines():
        t = ln.split()
        if t[0] == "centre":
            cur = {"centre": np.array(t[1:], np.float32), "beads": []}
            blocks.append(cur)
        elif t[0] == "quat":
            cur["quat"] = np.array([float(x) for x in t[1:]])
        else:
            cur["beads"].append([int(t[1])] + [float(x) for x in t[2:]])
    for b in blocks:
        a = np.array(b["beads"], np.float64)
        b["types"] = a[:, 0].astype(int)
        b["pos"] = a[:, 1:4].astype(np.float32)
        b["rel"] = a[:, 4:7].astype(np.float32)
    return blocks


@pytest.fixture(scope="module")
def inputs(tmp_path_factory, built_lib):
    d = str(tmp_path_factory.mktemp("facade"))
    w = synth.crowded(5)
    synth.write_reference_inputs(w, 0, d, 100, 2, 2, sample_frequency=50)
    return d


def test_moves_match_python_model(inputs):
    d = inputs
    aa, pp = os.path.join(d, "data", "AminoAcids"), os.path.join(d, "data", "pair_potentials_MJ1996")
    pdb = os.path.join(d, "pdb", "chain000.pdb")
    blocks = _parse_blocks(_check("moves", aa, pp, pdb))
    table = AminoAcidTable.load(aa)
    table.load_pairs(pp)
    m = Molecule.from_pdb(pdb, table)
    saved = m.copy()
    expect = [m.copy()]
    m.translate(np.array([1.25, -0.5, 3.0], np.float32))
    expect.append(m.copy())
    m.set_position(np.array([10.0, 20.0, 30.0], np.float32))
    expect.append(m.copy())
    m.rotate_q(normalise_axis(0.3, -0.4, 0.5), 0.7)
    expect.append(m.copy())
    expect.append(saved)
    assert len(blocks) == len(expect)
    for b, e in zip(blocks, expect):
        assert np.array_equal(b["types"], e.types)
        assert np.array_equal(b["pos"], e.pos)        # %.9g round-trips float32
        assert np.array_equal(b["rel"], e.rel)
        assert np.array_equal(b["centre"], e.centre)
        assert np.array_equal(b["quat"], e.quat)       # %.17g round-trips float64


def test_facade_exports_reference_method_names(built_lib):
    nm = shutil.which("nm")
    if nm is None:
        pytest.skip("nm not available")
    out = subprocess.run([nm, "-DC", "--defined-only", build.FACADE], capture_output=True,
                         text=True).stdout
    for sym in ("remc::Replica::E()", "remc::Replica::EonDevice()", "remc::Replica::MCSearch(int)",
                "remc::Replica::exchangeReplicas(remc::Replica&)",
                "remc::Replica::ReplicaDataToDevice()", "remc::Replica::ReplicaDataToHost()",
                "remc::Replica::MoleculeDataToDevice(int)", "remc::Replica::FreeDevice()",
                "remc::Replica::loadMolecule(char const*)",
                "remc::Replica::setLJpotentials(float const*)",
                "remc::Replica::copy(remc::Replica const&)",
                "remc::Molecule::initFromPDB(char const*)",
                "remc::Molecule::rotateQ(remc::Vector3double const&, double)",
                "remc::Molecule::undoStateChange(remc::Molecule const*)",
                "remc::AminoAcids::loadLJPotentialData(char const*)",
                "remc::ReplicaExchange::run(int, int)"):
        assert sym in out, sym


def test_missing_pdb_is_an_error_not_a_crash(inputs):
    d = inputs
    aa, pp = os.path.join(d, "data", "AminoAcids"), os.path.join(d, "data", "pair_potentials_MJ1996")
    r = subprocess.run([build.FACADE_CHECK, "moves", aa, pp, os.path.join(d, "nope.pdb")],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "error" in r.stderr
