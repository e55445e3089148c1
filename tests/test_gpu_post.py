"""GPU post-processing against the oracle and end to end: pose
reconstruction (remc_post_rebuild) bit-identical to pdbgen's arithmetic
(oracle_post_rebuild), DRMS (remc_post_drms) against the oracle's loop-order
sum, and the pdbgen and trajectory tools on engine output."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_rebuild_bit_identical_to_oracle(built_lib):
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import post
    from remcdockingsimulator_b200.model import Molecule
    rng = np.random.default_rng(3)
    sizes = [40, 33, 1, 1, 1]
    mols = []
    for k, n in enumerate(sizes):
        m = Molecule.from_beads(np.zeros(n, np.int32),
                                rng.normal(scale=6.0, size=(n, 3)) + 20.0 * k)
        mols.append(m)
    shift = [1, 1, 0, 0, 1]
    box = 90.0
    F = 7
    quat = rng.normal(size=(F, len(sizes), 4))
    centre = rng.uniform(-100, 200, size=(F, len(sizes), 3)).astype(np.float32)
    pos, cout = post.rebuild(mols, shift, box, quat, centre)
    rel0 = np.concatenate([m.rel for m in mols])
    ms = np.cumsum([0] + sizes).astype(np.int32)
    for f in range(F):
        ref = ob.post_rebuild(rel0, ms, shift, mols[0].centre, box, quat[f], centre[f])
        assert np.array_equal(pos[f], ref), f


def test_drms_matches_oracle(built_lib):
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import post
    rng = np.random.default_rng(5)
    ms = np.array([0, 50, 100, 150], np.int32)
    ref = rng.normal(scale=10.0, size=(150, 3)).astype(np.float32)
    frames = (ref[None] + rng.normal(scale=3.0, size=(6, 150, 3))).astype(np.float32)
    for reverse in (False, True):
        d, nat, rec, bind = post.drms(frames, ref, ms, reverse=reverse)
        for f in range(6):
            dr, cnt = ob.post_drms(frames[f], ref, ms, reverse, 12.0, 15.0)
            assert abs(d[f] - dr) <= 1e-12 * abs(dr), (f, d[f], dr)
            assert (nat[f], rec[f], bind[f]) == tuple(cnt)
    with pytest.raises(Exception):  # reverse order needs equal molecule lengths
        post.drms(frames, ref, np.array([0, 50, 150], np.int32), reverse=True)


def _placed_run(d, chain_ids, n_crowders, box_override=None):
    """Write placed PDBs of the crowded workload's chains and crowders, run
    the engine on them, and return (table, paths, flags, system, engine state)."""
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import Engine, make_params
    from remcdockingsimulator_b200.model import Molecule, System, write_pdb_ca
    s0 = synth.crowded(5).systems[0]
    table = s0.table
    os.makedirs(os.path.join(d, "data"), exist_ok=True)
    table.write(os.path.join(d, "data", "AminoAcids"))
    table.write_pairs(os.path.join(d, "data", "pair_potentials_MJ1996"))
    chains = [m for m in s0.molecules if not m.crowder]
    crowders = [m for m in s0.molecules if m.crowder][:n_crowders]
    paths, flags, mols = [], [], []
    for k, m in enumerate([chains[i] for i in chain_ids] + crowders):
        p = os.path.join(d, "m%03d.pdb" % k)
        off = np.array([45.0 * k, 0.0, 0.0], np.float32) if not m.crowder else 0.0
        write_pdb_ca(p, np.zeros(m.n, np.int32) if m.crowder else m.types,
                     (m.pos + off).astype(np.float32), table)
        mm = Molecule.from_pdb(p, table)
        mm.crowder = m.crowder
        paths.append(p)
        flags.append(m.crowder)
        mols.append(mm)
    box = box_override or s0.box
    s = System(mols, box, table)
    R = 4
    with Engine([s], R, make_params()) as eng:
        eng.set_replica_params([np.full(R, 300.0, np.float32)], np.full(R, 2.0, np.float32),
                               np.full(R, 0.3))
        eng.energy_full()
        eng.sweep(800, 99, 0)
        st = eng.download_state()
        en = eng.energies()
        slices = eng.instance_slices()
    return table, paths, flags, s, st, en, slices


def test_pdbgen_end_to_end(tmp_path, built_lib):
    from remcdockingsimulator_b200 import post
    from remcdockingsimulator_b200.model import read_pdb_ca
    d = str(tmp_path)
    table, paths, flags, s, st, en, slices = _placed_run(d, [0, 1], 6)
    pos, rel, cen, quat = st
    base = os.path.join(d, "run_repulsive_1_")
    with open(base + "fileindex", "w") as fh:
        fh.write("index molecule_file_path crowder(Y/N)\n")
        for i, (p, c) in enumerate(zip(paths, flags)):
            fh.write("%2d %s %s\n" % (i, p, "Y" if c else "N"))
    with open(base + "boundconformations", "w") as fh:
        fh.write("# iteration; complex free energy (replica free energy); temperature;\n")
        fh.write("# molecule: rotation(w,x,y,z) position(x,y,z) 1 line per other molecule\n")
        for k, (bs, msl) in enumerate(slices):
            fh.write("%d; %0.5f (%0.5f); %0.1f\n" % (20_000_000 + k, en[k] - 1.0, en[k], 300.0))
            for i, m in enumerate(range(msl.start, msl.stop)):
                fh.write("%d %2d: %f %f %f %f %f %f %f\n" % ((1 if flags[i] else 0, i) +
                                                           tuple(quat[m]) + tuple(cen[m])))
    out = os.path.join(d, "pdbgen_results")
    summ = post.pdbgen(base + "fileindex", s.box, data_dir=os.path.join(d, "data"), out_dir=out,
                       log=lambda *_: None)
    assert summ["kept"] == len(slices) and len(summ["files"]) == len(slices)
    n_chain = sum(m.n for m, c in zip(s.molecules, flags) if not c)
    for k, (bs, msl) in enumerate(slices):
        got = summ["positions"][k]
        want = pos[bs][:n_chain]
        diff = got - want
        diff -= s.box * np.round(diff / s.box)  # pdbgen moves chains by whole boxes
        assert np.abs(diff).max() < 2e-3, (k, np.abs(diff).max())  # poses were written at %f
        types, xyz = read_pdb_ca(summ["files"][k], table)
        assert types.shape[0] == n_chain and np.abs(xyz - got).max() < 1e-3
    # the DRMS written to drms.dat is the oracle's DRMS of the rebuilt frames
    from oracle import bindings as ob
    ms = np.cumsum([0] + [m.n for m, c in zip(s.molecules, flags) if not c]).astype(np.int32)
    ref = np.concatenate([m.pos for m, c in zip(s.molecules, flags) if not c])
    dat = np.loadtxt(base + "drms.dat", ndmin=2)
    for k in range(len(slices)):
        dr, _ = ob.post_drms(summ["positions"][k], ref, ms)
        assert abs(summ["drms"][k] - dr) <= 1e-12 * dr
        assert abs(dat[k, 1] - dr) <= 1e-6 * dr


def test_trajectory_tool(tmp_path, built_lib):
    from remcdockingsimulator_b200 import post
    from remcdockingsimulator_b200.engine import Engine, make_params
    from oracle import bindings as ob
    d = str(tmp_path)
    # a homodimer: the same chain twice (reverse-order DRMS needs equal lengths)
    table, paths, flags, s, st, en, slices = _placed_run(d, [0, 0], 0, box_override=200.0)
    pos = st[0]
    traj = os.path.join(d, "traj.pdb")
    lengths = [m.n for m in s.molecules]
    with open(traj, "w") as fh:
        for k, (bs, msl) in enumerate(slices):
            fh.write("MODEL%9d\n" % (k + 1))
            for b, x in enumerate(pos[bs]):
                t = s.molecules[0 if b < lengths[0] else 1].types[b % lengths[0]]
                fh.write("ATOM  %5d  CA  %3s A%4d    %8.3f%8.3f%8.3f  1.00  1.00\n" % (
                    b + 1, table.snames[int(t)].upper(), b + 1, x[0], x[1], x[2]))
            fh.write("ENDMDL\n")
    lst = os.path.join(d, "processTraj.exp")
    with open(lst, "w") as fh:
        fh.write("\n".join(paths) + "\n")
    res = post.process_trajectory(traj, lst, lengths, box=s.box, data_dir=os.path.join(d, "data"),
                                  log=lambda *_: None)
    assert res["frames"] == len(slices)
    frames, _ = post.read_trajectory(traj, lengths, table)
    ref = np.concatenate([m.pos for m in s.molecules])
    ms = np.cumsum([0] + lengths).astype(np.int32)
    for k in range(len(slices)):
        dr, _ = ob.post_drms(frames[k], ref, ms, reverse=True)
        assert abs(res["drms"][k] - dr) <= 1e-12 * dr
        o = ob.FP64Oracle(s, make_params())
        e_ref = o.energy(frames[k])
        assert abs(res["energies"][k] - e_ref) <= 1e-5 * max(abs(e_ref), 1e-3)
    lines = open(traj + ".drms.dat").read().split()
    assert len(lines) == 2 * len(slices)
    assert open(traj + ".delim.pdb").read().count("ENDMDL") == len(slices)
