"""GPU tests of Replica::sample on the device and of the REMC driver."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_RTOL = 1e-5


def _oracle_chunks(o, s, state, T, ts, rs, seed, slot, n_steps, f, e0, thr):
    """Oracle MC in chunks of f steps; returns per-chunk (E_nc, bound, state)."""
    out = []
    E = e0
    for c in range(n_steps // f):
        state, E, flags, mol, dE, cnt = o.mc_run(state, T, ts, rs, seed, c * f, slot, 0, f, E)
        ecc = o.noncrowder_pair_energy(state[0])
        has_crowders = any(m.crowder for m in s.molecules)
        enc = E + ecc if has_crowders else E
        out.append((enc, enc < thr, [a.copy() for a in state]))
    return out, state, E


@pytest.mark.parametrize("name,cluster", [("crowded", 1), ("two_chain", 1), ("crowded", 4)])
def test_sampling_counts_and_bound_decisions(name, cluster, built_lib):
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import Engine
    w = synth.WORKLOADS[name](17)
    s = w.systems[0]
    R, n, f, seed = 3, 600, 50, 99
    lad = w.ladders[0][:R]
    o = ob.FP64Oracle(s, w.params)
    e_full0 = o.energy(s.state()[0])
    ecc0 = o.noncrowder_pair_energy(s.state()[0])
    # a threshold near the middle of the trajectory's E_nc so both outcomes occur
    probe, _, _ = _oracle_chunks(o, s, s.state(), float(lad[0]), 0.5, 0.2, seed, 0, n, f,
                                 e_full0, 1e30)
    thr = float(np.median([p[0] for p in probe]))
    with Engine([s], R, w.params) as eng:
        eng.set_replica_params([lad], np.full(R, 0.5, np.float32), np.full(R, 0.2))
        if cluster > 1:
            eng.set_cluster(cluster)  # rank 0 of each cluster writes the samples
        e0 = eng.energy_full()
        assert abs(eng.noncrowder_energies()[0] - ecc0) <= E_RTOL * max(abs(ecc0), 1e-3)
        eng.set_sampling(f, 0, thr, max_records=R * n // f, max_poses=R * n // f * s.n_mol)
        eng.sweep(n, seed, 0)
        n_s, n_b = eng.sample_counters()
        recs, poses, dropped = eng.read_samples()
        ecc_gpu = eng.noncrowder_energies()
        st = eng.download_state()
        sl = eng.instance_slices()
    assert dropped == 0
    assert np.all(n_s == n // f)
    for k in range(R):
        chunks, fin, E = _oracle_chunks(o, s, s.state(), float(lad[k]), 0.5, 0.2, seed, k, n, f,
                                        float(e0[k]), thr)
        assert n_b[k] == sum(1 for c in chunks if c[1]), (k, n_b[k])
        ecc_ref = o.noncrowder_pair_energy(fin[0])
        assert abs(ecc_gpu[k] - ecc_ref) <= E_RTOL * max(abs(ecc_ref), 1e-3)
        mine = sorted([r for r in recs if r["inst"] == k], key=lambda r: r["label"])
        bound_chunks = [(i, c) for i, c in enumerate(chunks) if c[1]]
        assert len(mine) == len(bound_chunks)
        for r, (i, c) in zip(mine, bound_chunks):
            assert r["label"] == i * f  # the chunk's start step, as the reference labels it
            assert abs(r["e_noncrowder"] - c[0]) <= E_RTOL * max(abs(c[0]), 1e-3)
            p = poses[r["pose_offset"]:r["pose_offset"] + r["n_mol"]]
            assert np.array_equal(p[:, :4], c[2][3])          # quaternions, bit-exact
            assert np.array_equal(p[:, 4:].astype(np.float32), c[2][2])  # centres


def test_driver_writes_reference_output_files(tmp_path, built_lib):
    from remcdockingsimulator_b200 import remc, synth
    from remcdockingsimulator_b200.model import AminoAcidTable
    w = synth.crowded(5)
    d = str(tmp_path)
    cfg = synth.write_reference_inputs(w, 0, d, 400, 4, 4, sample_frequency=50)
    table = AminoAcidTable.load(os.path.join(d, "data", "AminoAcids"))
    table.load_pairs(os.path.join(d, "data", "pair_potentials_MJ1996"))
    a = remc.parse_cli(["-f", cfg, "-r", "6", "--seed", "3", "--output-dir",
                        os.path.join(d, "output")])
    a.pid = 4242
    mols = remc.load_config(a, table, log=lambda *_: None)
    remc.parse_cli(["-f", cfg, "-r", "6"], a)  # flags override the file, as main() does
    a.sample_after = 0
    a.sensitivity = True
    remc.write_file_index(a)
    from remcdockingsimulator_b200.model import System
    summary = remc.simulate(a, System(mols, a.bound, table), log=lambda *_: None)
    base = summary["files"]
    fb = open(base + "_fractionBound").read().splitlines()
    ar = open(base + "_acceptance_ratios").read().splitlines()
    ex = open(base + "_exchange_freq").read().splitlines()
    assert fb[0] == "# Fraction Bound" and fb[2].startswith("Iteration:  290.0Ki 290.0Kc")
    # resteps - 1 exchange rounds, each reported, plus the final line
    assert len([l for l in fb if l.strip().endswith(" ") or "|" in l]) == 4
    assert len(ex) == 1 + 3 and ex[1].split()[0] == "1"
    assert all(l.count("|") == 6 for l in ar[3:])
    idx = open(os.path.join(d, "output", "synth_repulsive_4242_fileindex")).read().splitlines()
    assert idx[0] == "index molecule_file_path crowder(Y/N)" and idx[-1].endswith(" Y")
    assert summary["replica_steps"] == 6 * 400
    # fluctuation sensitivities: one row per temperature, one sample per
    # replica per sampling chunk (2 chunks of 50 steps per 100-step block);
    # the total is the covariance term plus the threshold term
    sens = open(base + "_sensitivity").read().splitlines()[1:]
    assert len(sens) == 6
    assert sum(int(l.split()[1]) for l in sens) == 6 * 4 * 2
    for l in sens:
        v = [float(x) for x in l.split()]
        if int(v[1]) > 0:
            assert all(np.isfinite(v[4:]))
            assert abs(v[6] - (v[4] + v[5])) <= 1e-5 * max(abs(v[6]), 1e-6)
