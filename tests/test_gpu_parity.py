"""GPU parity: the CUDA engine against the FP64 oracle and the reference's own
CPU engine, through the C ABI (ctypes). Tolerances: energies <= 1e-5 relative
(FP32 pair terms, FP64 sums); move arithmetic bit-exact; accept/reject
decisions identical."""
import math

import numpy as np
import pytest

from conftest import golden_system

pytestmark = pytest.mark.gpu

E_RTOL = 1e-5


def _engine(systems, R, params):
    from remcdockingsimulator_b200.engine import Engine
    return Engine(systems, R, params)


def test_energy_full_golden_structures(golden, golden_table, built_lib):
    """GPU full energy of the 10 golden structures vs the reference's own
    Replica::E() values (one system each, one launch)."""
    from remcdockingsimulator_b200.engine import make_params
    systems = [golden_system(golden, golden_table, k) for k in range(10)]
    with _engine(systems, 1, make_params()) as eng:
        e = eng.energy_full()
    for k, st in enumerate(golden["structures"]):
        ref = st["reference_E"]
        if abs(ref) > 1e-2:
            assert abs(e[k] - ref) / abs(ref) < E_RTOL, (k, e[k], ref)
        else:
            assert abs(e[k] - ref) < 1e-6, (k, e[k], ref)


@pytest.mark.parametrize("name,mode", [("two_chain", 1), ("crowded", 1), ("crowded", 0)])
def test_energy_full_vs_oracle(name, mode, built_lib):
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import make_params
    w = synth.WORKLOADS[name](11)
    p = w.params if mode == 1 else make_params(lambda_=0.16)
    s = w.systems[0]
    with _engine([s], 2, p) as eng:
        e = eng.energy_full()
    ref = ob.FP64Oracle(s, p).energy(s.state()[0])
    assert e[0] == e[1]
    assert abs(e[0] - ref) <= E_RTOL * max(abs(ref), 1e-3), (e[0], ref)


def test_energy_full_uneven_batch_vs_oracle(built_lib):
    """Several systems of uneven size in one handle (one persistent launch)."""
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    rng = np.random.default_rng(5)
    table = synth.contact_table(rng)
    systems = [synth.build_system(rng, table, [int(rng.integers(20, 200)) for _ in range(k)],
                                  int(rng.integers(0, 300)), 12.0, 160.0 + 20 * k)
               for k in (2, 3, 5, 8)]
    p = synth.benchmark_params()
    with _engine(systems, [3, 1, 2, 4], p) as eng:
        e = eng.energy_full()
        first = eng.inst_first
    for i, s in enumerate(systems):
        ref = ob.FP64Oracle(s, p).energy(s.state()[0])
        assert abs(e[first[i]] - ref) <= E_RTOL * max(abs(ref), 1e-3), (i, e[first[i]], ref)


def test_delta_energy_api_vs_oracle(built_lib):
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    w = synth.crowded(2)
    s = w.systems[0]
    o = ob.FP64Oracle(s, w.params)
    pos = s.state()[0]
    ms = s.topology()[0]
    with _engine([s], 1, w.params) as eng:
        for m in (0, 1, 2, 250, 401):
            new = (pos[ms[m]:ms[m + 1]] + np.array([1.3, -0.4, 2.2], np.float32)).astype(np.float32)
            d_gpu = eng.delta_energy(0, m, new)
            d_ref = o.energy_molecule(pos, m, new) - o.energy_molecule(pos, m, pos[ms[m]:ms[m + 1]])
            scale = abs(o.energy_molecule(pos, m, new)) + abs(
                o.energy_molecule(pos, m, pos[ms[m]:ms[m + 1]]))
            assert abs(d_gpu - d_ref) <= E_RTOL * max(scale, 1e-3), (m, d_gpu, d_ref)


def _run_sweep_vs_oracle(w, R, n_steps, seed, step0=0, tsteps=None, rsteps=None, cluster=1,
                         beads_shared=True):
    from oracle import bindings as ob
    s = w.systems[0]
    lad = w.ladders[0][:R]
    ts = np.full(R, w.translate_step, np.float32) if tsteps is None else tsteps
    rs = np.full(R, w.rotate_step) if rsteps is None else rsteps
    with _engine([s], R, w.params) as eng:
        eng.set_replica_params([lad], ts, rs)
        if cluster > 1:
            eng.set_cluster(cluster)
            assert eng.schedule()[2] == cluster
        if not beads_shared:
            eng.set_bead_storage(False)
            assert not eng.beads_in_shared_memory()
        e0 = eng.energy_full()
        eng.sweep(n_steps, seed, step0)
        e_run = eng.energies()
        st = eng.download_state()
        e_full = eng.energy_full()
        acc, accA, rej = eng.counters()
        slices = eng.instance_slices()
    o = ob.FP64Oracle(s, w.params)
    for k in range(R):
        (pos, rel, cen, quat), E, flags, mol, dE, cnt = o.mc_run(
            s.state(), float(lad[k]), float(ts[k]), float(rs[k]), seed, step0, k, 0, n_steps,
            float(e0[k]), energy_mode=0)
        bs, msl = slices[k]
        assert (acc[k], accA[k], rej[k]) == cnt, (k, (acc[k], accA[k], rej[k]), cnt)
        assert np.array_equal(st[0][bs], pos), k
        assert np.array_equal(st[1][bs], rel), k
        assert np.array_equal(st[2][msl], cen), k
        assert np.array_equal(st[3][msl], quat), k
        scale = max(np.abs(dE).sum(), abs(E), 1e-3)
        assert abs(e_run[k] - E) <= E_RTOL * scale, (k, e_run[k], E)
        ref_full = o.energy(pos)
        assert abs(e_full[k] - ref_full) <= E_RTOL * max(abs(ref_full), 1e-3)
    return e_run, e_full


def test_sweep_two_chain_vs_oracle(built_lib):
    from remcdockingsimulator_b200 import synth
    w = synth.two_chain(7)
    tr = np.linspace(0.5, 3.0, 4).astype(np.float32)
    rr = np.linspace(0.1, 0.5, 4)
    _run_sweep_vs_oracle(w, 4, 600, seed=2024, step0=17, tsteps=tr, rsteps=rr)


def test_sweep_crowded_vs_oracle(built_lib):
    from remcdockingsimulator_b200 import synth
    w = synth.crowded(7)
    _run_sweep_vs_oracle(w, 3, 1500, seed=77)


@pytest.mark.parametrize("cluster", [2, 4, 8])
def test_sweep_cluster_vs_oracle(cluster, built_lib):
    """A replica spread over a cluster of CTAs (pair loops split over the
    cluster, partial sums exchanged through distributed shared memory) follows
    the oracle's trajectory like a single CTA does."""
    from remcdockingsimulator_b200 import synth
    w = synth.crowded(7)
    _run_sweep_vs_oracle(w, 3, 1500, seed=77, cluster=cluster)
    w2 = synth.two_chain(7)
    _run_sweep_vs_oracle(w2, 2, 800, seed=5, cluster=cluster)


def test_sweep_crowded_reference_mode_rotating_crowders(built_lib):
    """Reference semantics: (6/r)^6 crowders with the 15 A cutoff, crowders are
    also rotated (a no-op move that is always accepted)."""
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import make_params
    w = synth.crowded(8)
    w.systems[0].translate_only_crowders = False
    w.params = make_params(lambda_=0.159)
    _run_sweep_vs_oracle(w, 2, 1200, seed=5)


def test_sweep_vs_reference_engine_bitwise(built_lib):
    """GPU sweep vs the reference's own Replica::MCSearch fed the same Philox
    stream: identical coordinates, rotations and decisions."""
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import make_params
    if not ob.reference_available():
        pytest.skip("reference harness not built")
    w = synth.two_chain(21)
    s = w.systems[0]
    p = make_params()  # the reference's compile-time constants
    n, seed, T, ts, rs = 500, 31337, 320.0, 1.0, 0.25
    with _engine([s], 1, p) as eng:
        eng.set_replica_params([np.array([T], np.float32)], [ts], [rs])
        eng.energy_full()
        eng.sweep(n, seed, 0)
        st = eng.download_state()
        e_gpu = eng.energies()[0]
    r = ob.ReferenceReplica(s, temperature=T)
    r.set_steps(ts, rs)
    u = np.stack([ob.step_uniforms(seed, t, 0, 0) for t in range(n)])
    flags, mol, en, under = r.mcsearch(u)
    assert under == 0
    sr = r.state()
    for a, b in zip(sr, st):
        assert np.array_equal(a, b)
    assert abs(e_gpu - en[-1]) <= E_RTOL * max(abs(en[-1]), 1e-3)


def test_sweep_plain_matches_persistent(built_lib):
    from remcdockingsimulator_b200 import synth
    w = synth.crowded(4)
    s = w.systems[0]
    R = 3
    outs = []
    for plain in (False, True):
        with _engine([s], R, w.params) as eng:
            eng.set_replica_params([w.ladders[0][:R]], np.full(R, 0.5, np.float32),
                                   np.full(R, 0.2))
            eng.energy_full()
            (eng.sweep_plain if plain else eng.sweep)(60, 99, 5)
            outs.append((eng.download_state(), eng.energies(), eng.counters()))
    for a, b in zip(outs[0][0], outs[1][0]):
        assert np.array_equal(a, b)
    assert np.array_equal(outs[0][1], outs[1][1])
    for a, b in zip(outs[0][2], outs[1][2]):
        assert np.array_equal(a, b)


def test_exchange_vs_oracle(built_lib):
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    w = synth.two_chain(3)
    s = w.systems[0]
    R = 8
    lad = np.linspace(290, 450, R).astype(np.float32)
    with _engine([s], R, w.params) as eng:
        eng.set_replica_params([lad], np.linspace(0.5, 4.0, R).astype(np.float32),
                               np.full(R, 0.2))
        eng.energy_full()
        eng.sweep(300, 1, 0)
        tos = np.arange(R, dtype=np.int32)
        sot = np.arange(R, dtype=np.int32)
        for rnd in range(6):
            en = eng.energies()
            eng.exchange(1234, rnd, rnd & 1)
            got = eng.temperature_map()
            n, tos, sot, acc = ob.exchange_round(lad, en, tos, sot, rnd & 1, 1234, rnd, 0)
            assert np.array_equal(got, tos), (rnd, got, tos)
            eng.sweep(100, 1, 300 + 100 * rnd)


@pytest.mark.parametrize("cluster", [1, 4])
def test_graph_run_matches_stepwise(cluster, built_lib):
    """remc_run (captured graph, device-side counters) == explicit
    sweep/exchange calls with the same counters (single CTAs, and clusters
    launched inside the captured graph)."""
    from remcdockingsimulator_b200 import synth
    w = synth.crowded(9)
    s = w.systems[0]
    R = 4
    lad = w.ladders[0][:R]
    res = []
    for graph in (True, False):
        with _engine([s, s], [R, R], w.params) as eng:
            eng.set_replica_params([lad, lad], np.full(2 * R, 0.5, np.float32),
                                   np.full(2 * R, 0.2))
            if cluster > 1:
                eng.set_cluster(cluster)
            eng.energy_full()
            if graph:
                eng.run(5, 200, 4242, 0, 0)
                eng.sync()
            else:
                for b in range(5):
                    eng.sweep(200, 4242, 200 * b)
                    eng.exchange(4242, b, b & 1)
            res.append((eng.download_state(), eng.energies(), eng.temperature_map()))
    for a, b in zip(res[0][0], res[1][0]):
        assert np.array_equal(a, b)
    assert np.array_equal(res[0][1], res[1][1])
    assert np.array_equal(res[0][2], res[1][2])


def test_energy_drift_after_long_sweep(built_lib):
    """The running energy (sum of FP64-reduced dE) stays within 1e-5 of a full
    recomputation after 5000 steps."""
    from remcdockingsimulator_b200 import synth
    w = synth.crowded(12)
    s = w.systems[0]
    with _engine([s], 4, w.params) as eng:
        eng.set_replica_params([w.ladders[0][:4]], np.full(4, 0.5, np.float32), np.full(4, 0.2))
        eng.energy_full()
        eng.sweep(5000, 8, 0)
        run = eng.energies()
        full = eng.energy_full()
    assert np.all(np.abs(run - full) <= 1e-5 * np.maximum(np.abs(full), 1.0)), (run, full)


def test_bad_inputs_are_rejected(built_lib):
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200._capi import RemcError
    w = synth.two_chain(1)
    s = w.systems[0]
    with _engine([s], 2, w.params) as eng:
        pos, rel, cen, quat = [np.concatenate([a, a]) for a in s.state()]
        before = eng.download_state()
        bad = pos.copy()
        bad[3, 1] = np.nan
        with pytest.raises(RemcError, match="non-finite"):
            eng.upload_state(bad, rel, cen, quat)
        badc = cen.copy()
        badc[1, 0] = np.inf
        with pytest.raises(RemcError, match="centre"):
            eng.upload_state(pos, rel, badc, quat)
        # a refused upload leaves the state as it was
        for a, b in zip(before, eng.download_state()):
            assert np.array_equal(a, b)
        with pytest.raises(RemcError):
            eng.sweep(10, 1, 0)  # replica parameters not set yet
        with pytest.raises(RemcError):
            eng.set_replica_params([np.array([300.0, 290.0], np.float32)], [0.5, 0.5], [0.2, 0.2])


def test_autotune_restores_state_and_schedules_agree(built_lib):
    """The autotuner leaves the state untouched, and every schedule gives the
    same trajectory."""
    from remcdockingsimulator_b200 import synth
    w = synth.crowded(14)
    s = w.systems[0]
    R = 4
    outs = []
    for sched in ("tuned", (128, True), (256, False), (64, True)):
        with _engine([s], R, w.params) as eng:
            eng.set_replica_params([w.ladders[0][:R]], np.full(R, 0.5, np.float32),
                                   np.full(R, 0.2))
            eng.energy_full()
            before = eng.download_state()
            e_before = eng.energies()
            if sched == "tuned":
                t, m, ms = eng.autotune(probe_steps=64)
                assert t in (128, 256) and ms > 0
                after = eng.download_state()
                for a, b in zip(before, after):
                    assert np.array_equal(a, b)
                assert np.array_equal(e_before, eng.energies())
                assert all(c.sum() == 0 for c in eng.counters())
            else:
                eng.set_schedule(*sched)
                with pytest.raises(Exception):
                    eng.set_schedule(96, True)  # thread counts are powers of two
                eng.set_schedule(*sched)
            eng.sweep(400, 11, 0)
            outs.append((eng.download_state(), eng.energies()))
    for o in outs[1:]:
        for a, b in zip(outs[0][0], o[0]):
            assert np.array_equal(a, b)
        assert np.allclose(outs[0][1], o[1], rtol=1e-9, atol=1e-9)
