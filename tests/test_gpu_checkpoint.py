"""Checkpoint/resume of the REMC driver on the GPU: a run resumed from a
checkpoint taken after exchange round 2 of 4 ends with the same conformations,
energies, temperature map and byte-identical output files as the run that
was never interrupted (saveSimulation layout, main.cpp:89-117, plus the exact
engine state)."""
import os
import shutil

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(d, pid):
    from remcdockingsimulator_b200 import remc, synth
    from remcdockingsimulator_b200.model import AminoAcidTable, System
    w = synth.crowded(9)
    cfg = synth.write_reference_inputs(w, 0, d, 800, 4, 4, sample_frequency=50)
    table = AminoAcidTable.load(os.path.join(d, "data", "AminoAcids"))
    table.load_pairs(os.path.join(d, "data", "pair_potentials_MJ1996"))
    a = remc.parse_cli(["-f", cfg, "-r", "8", "--seed", "11"])
    a.pid = pid
    mols = remc.load_config(a, table, log=lambda *_: None)
    remc.parse_cli(["-f", cfg, "-r", "8"], a)
    a.sample_after = 0
    return a, System(mols, a.bound, table)


def _files(out_dir, base):
    names = ("_fractionBound", "_boundconformations", "_acceptance_ratios", "_exchange_freq")
    return {n: open(os.path.join(out_dir, base + n), "rb").read() for n in names}


def test_resume_continues_bit_for_bit(tmp_path, built_lib):
    from remcdockingsimulator_b200 import remc
    d = str(tmp_path)
    quiet = dict(log=lambda *_: None)

    # A: straight through
    a, s = _setup(d, 777)
    a.output_dir = os.path.join(d, "A")
    ref = remc.simulate(a, s, **quiet)

    # B: checkpoint after every exchange round; snapshot files after round 2
    a, s = _setup(d, 777)
    a.output_dir = os.path.join(d, "B")
    a.checkpoint_every = a.mcsteps // a.resteps
    a.checkpoint_dir = os.path.join(d, "ckB")
    snap = os.path.join(d, "C")

    def hook(path, blocks):
        if blocks == 2:
            os.makedirs(os.path.join(snap, "ck"), exist_ok=True)
            shutil.copy(path, os.path.join(snap, "ck", os.path.basename(path)))
            shutil.copy(path + ".state.npz", os.path.join(snap, "ck", os.path.basename(path) +
                                                          ".state.npz"))
            for fn in os.listdir(a.output_dir):
                shutil.copy(os.path.join(a.output_dir, fn), os.path.join(snap, fn))
    full = remc.simulate(a, s, on_checkpoint=hook, **quiet)

    # C: resume from the round-2 checkpoint into the snapshot of the files
    ck = os.path.join(snap, "ck", "synth_repulsive_777")
    hdr = remc.read_checkpoint_header(ck)
    assert hdr["pid"] == 777 and hdr["current_step"] == 2 * (800 // 4)
    a, s = _setup(d, 777)
    a.output_dir = snap
    a.resume = ck
    res = remc.simulate(a, s, **quiet)

    for other in (full, res):
        assert np.array_equal(other["energies"], ref["energies"])
        assert np.array_equal(other["temperature_of_slot"], ref["temperature_of_slot"])
    base = "synth_repulsive_777"
    fa = _files(os.path.join(d, "A"), base)
    assert _files(os.path.join(d, "B"), base) == fa
    assert _files(snap, base) == fa
