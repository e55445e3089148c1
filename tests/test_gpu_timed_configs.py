"""GPU parity on the configurations the benchmark times, built exactly as
bench.py builds them, against the FP64 oracle:

  two_chain  config 0 at its stated 20 replicas (290-450 K), 1000 steps
  crowded    config 1 at its 32 replicas, 1000 steps
  batch64    config 2: all 64 systems and 1024 replicas under the schedule
             remc_autotune picks; the full energy of every system, and
             1000-step trajectories of 8 systems (the smallest, the largest,
             the most crowded, the least crowded, the one with most chains,
             the one with the longest chain and two others) at their coldest
             and hottest replica
  assembly   config 4: 60 x 150-residue chains + 2000 crowders (11,000 beads,
             59.8M pairs), 32 replicas on clusters of 4 CTAs with the beads in
             shared memory; the full energy, and 300-step trajectories of two
             replicas

Tolerances: energies within 1e-5 relative (FP32 pair terms, FP64 sums);
coordinates, rotations and accept counters bit-identical.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_RTOL = 1e-5


def _close(a, b, scale=None):
    s = max(abs(b), 1e-3) if scale is None else scale
    return abs(a - b) <= E_RTOL * s


def _follow(eng, w, o_of, picks, n_steps, seed, step0, e0):
    """Compare the engine's state after a sweep with the oracle's trajectory
    of each (system, slot) in picks, from the same start state."""
    st = eng.download_state()
    e_run = eng.energies()
    e_full = eng.energy_full()
    acc, accA, rej = eng.counters()
    slices = eng.instance_slices()
    ts = np.float32(w.translate_step)
    worst = 0.0
    for si, k in picks:
        inst = eng.inst_first[si] + k
        s = w.systems[si]
        o = o_of(si)
        (pos, rel, cen, quat), E, flags, mol, dE, cnt = o.mc_run(
            s.state(), float(w.ladders[si][k]), float(ts), float(w.rotate_step), seed, step0, k,
            si, n_steps, float(e0[inst]), energy_mode=0)
        bs, msl = slices[inst]
        assert (acc[inst], accA[inst], rej[inst]) == cnt, (si, k, (acc[inst], accA[inst],
                                                                   rej[inst]), cnt)
        assert np.array_equal(st[0][bs], pos), (si, k)
        assert np.array_equal(st[1][bs], rel), (si, k)
        assert np.array_equal(st[2][msl], cen), (si, k)
        assert np.array_equal(st[3][msl], quat), (si, k)
        scale = max(np.abs(dE).sum(), abs(E), 1e-3)
        assert _close(e_run[inst], E, scale), (si, k, e_run[inst], E)
        ref_full = o.energy(pos)
        assert _close(e_full[inst], ref_full), (si, k, e_full[inst], ref_full)
        worst = max(worst, abs(e_full[inst] - ref_full) / max(abs(ref_full), 1e-3))
    return worst


def _single_system(w, n_steps, seed, picks=None, cluster=1, beads_shared=None):
    from oracle import bindings as ob
    from remcdockingsimulator_b200.engine import Engine
    s = w.systems[0]
    R = w.n_replicas[0]
    with Engine(w.systems, w.n_replicas, w.params) as eng:
        eng.set_replica_params(w.ladders, np.full(1, w.translate_step, np.float32),
                               np.full(1, w.rotate_step))
        if cluster > 1:
            eng.set_cluster(cluster)
            assert eng.schedule()[2] == cluster
        if beads_shared is not None:
            assert eng.beads_in_shared_memory() == beads_shared
        e0 = eng.energy_full()
        o = ob.FP64Oracle(s, w.params)
        ref0 = o.energy(s.state()[0])
        assert np.all(e0 == e0[0])
        assert _close(e0[0], ref0), (e0[0], ref0)
        eng.sweep(n_steps, seed, 0)
        picks = picks if picks is not None else [(0, k) for k in range(R)]
        _follow(eng, w, lambda si: o, picks, n_steps, seed, 0, e0)


def test_two_chain_twenty_replicas_vs_oracle(built_lib):
    from remcdockingsimulator_b200 import synth
    w = synth.two_chain(0)
    assert w.n_replicas == [20]
    _single_system(w, 1000, seed=101)


def test_crowded_thirty_two_replicas_vs_oracle(built_lib):
    from remcdockingsimulator_b200 import synth
    w = synth.crowded(0)
    assert w.n_replicas == [32]
    _single_system(w, 1000, seed=102)


def test_assembly_clusters_of_four_vs_oracle(built_lib):
    """The 11,000-bead assembly in its benchmarked schedule: every replica on
    a cluster of 4 CTAs with the whole system in each CTA's shared memory."""
    from remcdockingsimulator_b200 import synth
    w = synth.assembly(0)
    assert w.systems[0].n_beads == 11000 and w.n_replicas == [32]
    _single_system(w, 300, seed=103, picks=[(0, 0), (0, 31)], cluster=4, beads_shared=True)


@pytest.fixture(scope="module")
def batch64():
    from remcdockingsimulator_b200 import synth
    return synth.batch64(0)


def _batch_picks(w):
    n_b = np.array([s.n_beads for s in w.systems])
    n_cr = np.array([sum(1 for m in s.molecules if m.crowder) for s in w.systems])
    n_ch = np.array([sum(1 for m in s.molecules if not m.crowder) for s in w.systems])
    longest = np.array([max(m.n for m in s.molecules if not m.crowder) for s in w.systems])
    chosen = []
    for si in (int(n_b.argmin()), int(n_b.argmax()), int(n_cr.argmax()), int(n_cr.argmin()),
               int(n_ch.argmax()), int(longest.argmax()), 17, 42):
        if si not in chosen:
            chosen.append(si)
    k = 0
    while len(chosen) < 8:
        if k not in chosen:
            chosen.append(k)
        k += 1
    return chosen


def test_batch64_all_systems_under_the_tuned_schedule_vs_oracle(batch64, built_lib):
    """batch64 exactly as the benchmark runs it: all 64 systems and their 1024
    replicas in one handle, the schedule chosen by remc_autotune."""
    from oracle import bindings as ob
    from remcdockingsimulator_b200.engine import Engine
    w = batch64
    assert len(w.systems) == 64 and w.n_inst == 1024
    oracles = {}

    def o_of(si):
        if si not in oracles:
            oracles[si] = ob.FP64Oracle(w.systems[si], w.params)
        return oracles[si]

    with Engine(w.systems, w.n_replicas, w.params) as eng:
        eng.set_replica_params(w.ladders, np.full(len(w.systems), w.translate_step, np.float32),
                               np.full(len(w.systems), w.rotate_step))
        e0 = eng.energy_full()
        before = eng.download_state()
        threads, smem, _ = eng.autotune(probe_steps=256)
        for a, b in zip(before, eng.download_state()):
            assert np.array_equal(a, b)
        # the full energy of every system
        for si, s in enumerate(w.systems):
            first = eng.inst_first[si]
            assert np.all(e0[first:first + w.n_replicas[si]] == e0[first])
            ref = o_of(si).energy(s.state()[0])
            assert _close(e0[first], ref), (si, e0[first], ref)
        seed, n_steps = 20241203, 1000
        eng.sweep(n_steps, seed, 0)
        picks = [(si, k) for si in _batch_picks(w) for k in (0, w.n_replicas[si] - 1)]
        assert len(picks) == 16
        _follow(eng, w, o_of, picks, n_steps, seed, 0, e0)
