"""Beads kept in global memory instead of shared memory (systems of any size):
the same trajectories bit for bit as the shared-memory sweep, single CTAs and
clusters; the oracle's trajectory; and a system too large for shared memory,
which remc_create schedules with global beads by itself."""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _digest(eng):
    h = hashlib.sha1()
    for x in eng.download_state():
        h.update(np.ascontiguousarray(x).tobytes())
    h.update(np.ascontiguousarray(eng.energies()).tobytes())
    for x in eng.counters():
        h.update(np.ascontiguousarray(x).tobytes())
    return h.hexdigest()


def _run(w, shared, cluster=1, steps=1500, seed=99):
    from remcdockingsimulator_b200.engine import Engine
    with Engine(w.systems, w.n_replicas, w.params) as eng:
        eng.set_replica_params(w.ladders, np.full(len(w.systems), w.translate_step, np.float32),
                               np.full(len(w.systems), w.rotate_step))
        if cluster > 1:
            eng.set_cluster(cluster)
        eng.set_bead_storage(shared)
        assert eng.beads_in_shared_memory() == shared
        eng.energy_full()
        eng.sweep(steps, seed, 0)
        return _digest(eng)


@pytest.mark.parametrize("name,cluster", [("crowded", 1), ("two_chain", 1), ("crowded", 2),
                                          ("two_chain", 4)])
def test_global_beads_bit_identical_to_shared(name, cluster, built_lib):
    from remcdockingsimulator_b200 import synth
    w = synth.WORKLOADS[name](12)
    assert _run(w, True, cluster) == _run(w, False, cluster)


def test_global_beads_bit_identical_on_a_batch(built_lib):
    from remcdockingsimulator_b200 import synth
    w = synth.batch64(3, n_systems=12)
    assert _run(w, True, steps=800) == _run(w, False, steps=800)


def test_global_beads_vs_oracle(built_lib):
    from test_gpu_parity import _run_sweep_vs_oracle
    from remcdockingsimulator_b200 import synth
    _run_sweep_vs_oracle(synth.crowded(7), 3, 1500, seed=77, beads_shared=False)
    _run_sweep_vs_oracle(synth.two_chain(7), 2, 800, seed=5, beads_shared=False, cluster=2)


def _large_system():
    """Two 60-residue chains near the centre of a 208 A box and about 17,400
    crowders (R = 3 A) on an 8 A lattice: about 17,500 beads, 280 KB of bead
    data, more than a CTA's shared memory."""
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.model import CROWDER_TYPE, Molecule, System
    rng = np.random.default_rng(5)
    table = synth.contact_table(rng)
    n_side, spacing = 26, 8.0
    box = n_side * spacing
    chains = []
    for k in range(2):
        xyz = synth.compact_chain(rng, 60) + np.array([box / 2 + 35.0 * k, box / 2, box / 2])
        chains.append(Molecule.from_beads(rng.integers(0, 20, 60), xyz))
    placed = np.concatenate([m.pos for m in chains]).astype(np.float64)
    g = (np.arange(n_side) + 0.5) * spacing
    sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    near = np.linalg.norm(sites[:, None, :] - placed[None, :, :], axis=-1).min(axis=1)
    crowders = []
    for p in sites[near > 8.0]:
        m = Molecule.from_beads([CROWDER_TYPE], p[None, :].astype(np.float32))
        m.crowder = True
        crowders.append(m)
    return System(chains + crowders, float(np.float32(box)), table, crowder_radius=3.0,
                  translate_only_crowders=True)


def test_system_too_large_for_shared_memory(built_lib):
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import Engine
    from remcdockingsimulator_b200.model import geometric_ladder
    s = _large_system()
    assert s.n_beads > 15000
    params = synth.benchmark_params()
    R = 2
    lad = geometric_ladder(300.0, 350.0, R)
    with Engine([s], R, params) as eng:
        assert not eng.beads_in_shared_memory()
        with pytest.raises(Exception):
            eng.set_bead_storage(True)  # does not fit
        assert not eng.beads_in_shared_memory()
        eng.set_replica_params([lad], np.full(R, 1.0, np.float32), np.full(R, 0.3))
        e0 = eng.energy_full()
        o = ob.FP64Oracle(s, params)
        ref0 = o.energy(s.state()[0])
        assert np.all(np.abs(e0 - ref0) <= 1e-5 * max(abs(ref0), 1e-3)), (e0, ref0)
        eng.sweep(400, 2024, 0)
        st = eng.download_state()
        acc, accA, rej = eng.counters()
        e_run = eng.energies()
        slices = eng.instance_slices()
    for k in range(R):
        (pos, rel, cen, quat), E, flags, mol, dE, cnt = o.mc_run(
            s.state(), float(lad[k]), 1.0, 0.3, 2024, 0, k, 0, 400, float(e0[k]), energy_mode=0)
        bs, msl = slices[k]
        assert (acc[k], accA[k], rej[k]) == cnt, (k, (acc[k], accA[k], rej[k]), cnt)
        assert np.array_equal(st[0][bs], pos), k
        assert np.array_equal(st[2][msl], cen), k
        assert abs(e_run[k] - E) <= 1e-5 * max(np.abs(dE).sum(), abs(E), 1e-3), (k, e_run[k], E)
