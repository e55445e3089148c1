"""GPU checks of the C++ Replica/Molecule facade against the Python engine and
the FP64 oracle on the same inputs: Replica::E, two Replica::MCSearch calls in
a row (bit-identical trajectory to the engine's sweep on the same Philox key),
and ReplicaExchange (bit-identical to Engine.run)."""
import os
import subprocess

import numpy as np
import pytest

from remcdockingsimulator_b200 import build, synth
from remcdockingsimulator_b200.model import Molecule, System, geometric_ladder, write_pdb_ca

pytestmark = pytest.mark.gpu
E_RTOL = 1e-5


def _check(*args):
    r = subprocess.run([build.FACADE_CHECK] + [str(a) for a in args], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r.stdout


@pytest.fixture(scope="module")
def placed(tmp_path_factory, built_lib):
    """Two chains and 40 crowders of the crowded workload written as placed
    PDBs; the Python side reads the same files."""
    d = str(tmp_path_factory.mktemp("facade_gpu"))
    s = synth.crowded(5).systems[0]
    table = s.table
    aa, pp = os.path.join(d, "AminoAcids"), os.path.join(d, "pairs")
    table.write(aa)
    table.write_pairs(pp)
    args, mols = [], []
    for k, m in enumerate(s.molecules[:42]):
        p = os.path.join(d, "m%03d.pdb" % k)
        write_pdb_ca(p, np.zeros(m.n, np.int32) if m.crowder else m.types, m.pos, table)
        args.append(("c:" if m.crowder else "") + p)
        mm = Molecule.from_pdb(p, table)
        mm.crowder = m.crowder
        mols.append(mm)
    return aa, pp, args, System(mols, s.box, table)


def _read_state(path):
    reps = []
    for ln in open(path):
        t = ln.split()
        if t[0] == "replica":
            reps.append({"label": int(t[1]), "T": np.float32(t[2]), "E": float(t[3]),
                         "cnt": tuple(int(x) for x in t[4:7]), "centre": [], "quat": [],
                         "pos": []})
        elif t[0] == "mol":
            reps[-1]["centre"].append([np.float32(x) for x in t[1:4]])
            reps[-1]["quat"].append([float(x) for x in t[4:8]])
        else:
            reps[-1]["pos"].append([np.float32(x) for x in t[1:4]])
    for r in reps:
        r["centre"] = np.array(r["centre"], np.float32)
        r["quat"] = np.array(r["quat"])
        r["pos"] = np.array(r["pos"], np.float32)
    return reps


def test_facade_energy_matches_engine_and_oracle(placed):
    from remcdockingsimulator_b200.engine import Engine
    from oracle import bindings as ob
    aa, pp, args, s = placed
    out = _check("energy", aa, pp, s.box, *args).split()
    e_fac, e_dev = float(out[0]), float(out[1])
    with Engine([s], 1) as eng:
        e_eng = float(eng.energy_full()[0])
    e_ref = ob.FP64Oracle(s, eng.params).energy(s.state()[0])
    assert e_fac == e_eng == e_dev
    assert abs(e_fac - e_ref) <= E_RTOL * max(abs(e_ref), 1e-3), (e_fac, e_ref)


def test_facade_mcsearch_matches_engine_sweep(placed, tmp_path):
    from remcdockingsimulator_b200.engine import Engine
    aa, pp, args, s = placed
    T, steps, seed = 320.0, 600, 97531
    outf = str(tmp_path / "mc.txt")
    out = _check("mc", aa, pp, s.box, T, steps, seed, outf, *args).split()
    got = _read_state(outf)[0]
    n1 = steps // 2
    with Engine([s], 1) as eng:
        # the facade's defaults: translate 0.5f, rotate 0.2f widened to double
        eng.set_replica_params([np.array([T], np.float32)], [np.float32(0.5)],
                               [float(np.float32(0.2))])
        e0 = eng.energy_full()[0]
        eng.sweep(n1, seed, 0)
        eng.energy_full()  # MCSearch restarts from the full energy of its conformation
        eng.sweep(steps - n1, seed, n1)
        pos, rel, cen, quat = eng.download_state()
        e1 = eng.energies()[0]
    assert float(out[0]) == e0
    assert float(out[1]) == e1
    assert np.array_equal(got["pos"], pos)
    assert np.array_equal(got["centre"], cen)
    assert np.array_equal(got["quat"], quat)
    assert sum(got["cnt"]) == steps


@pytest.mark.parametrize("cluster", [1, 2])
def test_facade_replica_exchange_matches_engine_run(placed, tmp_path, cluster, monkeypatch):
    from remcdockingsimulator_b200.engine import Engine
    aa, pp, args, s = placed
    R, blocks, steps, seed = 6, 3, 200, 424242
    tmin, tmax = 290.0, 480.0
    outf = str(tmp_path / "remc.txt")
    if cluster > 1:
        monkeypatch.setenv("REMC_CHECK_CLUSTER", str(cluster))
    _check("remc", aa, pp, s.box, R, tmin, tmax, blocks, steps, seed, outf, *args)
    got = _read_state(outf)
    lad = geometric_ladder(tmin, tmax, R)
    with Engine([s], R) as eng:
        eng.set_replica_params([lad], np.full(R, np.float32(0.5), np.float32),
                               np.full(R, float(np.float32(0.2))))
        if cluster > 1:
            eng.set_cluster(cluster)
        eng.energy_full()
        eng.run(blocks, steps, seed, 0, 0)
        pos, rel, cen, quat = eng.download_state()
        E = eng.energies()
        tmap = eng.temperature_map()
        slices = eng.instance_slices()
    assert len(got) == R
    for k in range(R):
        bs, ms = slices[k]
        assert got[k]["T"] == lad[tmap[k]]
        assert got[k]["label"] == int(tmap[k])   # labels follow the temperatures
        assert got[k]["E"] == E[k]
        assert np.array_equal(got[k]["pos"], pos[bs])
        assert np.array_equal(got[k]["quat"], quat[ms])
