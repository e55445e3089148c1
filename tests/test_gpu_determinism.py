"""Run-to-run determinism of the persistent sweep: the same inputs, seed and
schedule give bit-identical final states, energies and counters, however the
warps of a CTA (or the CTAs of a cluster) drift against one another.

The workloads are chosen to exercise the shared-memory buffers that warps
hand to one another without a barrier in between: a chains-only system
(consecutive rotations of different chains, whose trial relative positions
are written by the next step's owners while slower warps still install the
previous step's) over many replicas and long enough to cross many refills of
the proposal ring, and the 64-system batch with the default schedule."""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _chains_only():
    from remcdockingsimulator_b200 import synth
    rng = np.random.default_rng(11)
    table = synth.contact_table(rng)
    return synth.build_system(rng, table, [40, 40, 40, 30, 30, 20], 0, 0.0, 90.0)


def _digest(eng):
    h = hashlib.sha1()
    for x in eng.download_state():
        h.update(np.ascontiguousarray(x).tobytes())
    h.update(np.ascontiguousarray(eng.energies()).tobytes())
    for x in eng.counters():
        h.update(np.ascontiguousarray(x).tobytes())
    return h.hexdigest()


def _run(systems, reps, ladders, params, steps, cluster=1, chunk=1000):
    from remcdockingsimulator_b200.engine import Engine
    with Engine(systems, reps, params) as eng:
        eng.set_replica_params(ladders, np.full(len(systems), 1.0, np.float32),
                               np.full(len(systems), 0.4))
        if cluster > 1:
            eng.set_cluster(cluster)
        eng.energy_full()
        for k in range(0, steps, chunk):
            eng.sweep(min(chunk, steps - k), 31337, k)
        return _digest(eng)


@pytest.mark.parametrize("cluster", [1, 2])
def test_chains_only_runs_are_bit_identical(cluster, built_lib):
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import make_params
    s = _chains_only()
    R = 192
    lad = [synth.geometric_ladder(290.0, 600.0, R)]
    runs = {_run([s], R, lad, make_params(), 3000, cluster=cluster) for _ in range(3)}
    assert len(runs) == 1, runs


def test_chains_only_trajectory_vs_oracle(built_lib):
    """The deterministic result is also the oracle's: every move of a long
    run with frequent consecutive rotations of different chains."""
    from test_gpu_parity import _run_sweep_vs_oracle
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import make_params
    s = _chains_only()
    R = 3
    w = synth.Workload("chains_only", [s], [R], [synth.geometric_ladder(290.0, 600.0, R)],
                       1.0, 0.4, make_params(), 3000, 1000)
    _run_sweep_vs_oracle(w, R, 3000, seed=31337)


def test_batch64_runs_are_bit_identical(built_lib):
    from remcdockingsimulator_b200 import synth
    w = synth.batch64(0)
    runs = {_run(w.systems, w.n_replicas, w.ladders, w.params, 3000) for _ in range(2)}
    assert len(runs) == 1, runs


def test_work_order_does_not_change_results(built_lib):
    """The persistent sweep takes replicas in decreasing order of their block's
    proposal costs (block_cost_kernel + rank_kernel before every launch), or in
    the static order: every replica's trajectory is the same either way. A
    rank that was not a permutation would run some replica twice and another
    not at all."""
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import Engine
    w = synth.batch64(0)
    digests = []
    for by_cost in (True, False):
        with Engine(w.systems, w.n_replicas, w.params) as eng:
            eng.set_replica_params(w.ladders, np.full(len(w.systems), 1.0, np.float32),
                                   np.full(len(w.systems), 0.4))
            eng.set_work_order(by_cost)
            assert eng.work_order() == (by_cost, 4 if by_cost else 2)
            eng.energy_full()
            for k in range(0, 2000, 1000):
                eng.sweep(1000, 4242, k)
            eng.run(2, 500, 4242, 2000, 0)
            digests.append(_digest(eng))
    assert digests[0] == digests[1]
