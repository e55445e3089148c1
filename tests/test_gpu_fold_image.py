"""The sweep's folded minimum image (min(|d|, L - |d|) per axis, valid while
every bead pair the sweep can reach is less than 1.5 box lengths apart): the
per-system flag set at upload, equal to the bound recomputed here, on for the
usual workloads, off for a long chain in a tight box and for a centre
uploaded three boxes away; and the oracle's trajectory on both paths."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _host_flag(s, state=None):
    pos, rel, cen, quat = s.state() if state is None else state
    L = float(np.float32(s.box))
    R = 1.01 * np.sqrt((rel.astype(np.float64) ** 2).sum(axis=1)).max()
    lo = np.minimum(pos.min(axis=0), -R)
    hi = np.maximum(pos.max(axis=0), L + R)
    margin = 1.49 * L - (hi - lo)
    return int(np.all(margin >= 0)), float(np.min(np.abs(margin)))


def _tight_box(table=None):
    """A 120-residue chain stretched along x and a 30-residue chain in a 60 A
    box: beads far from their centre, so pairs can be more than 1.5 L apart."""
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.model import Molecule, System
    rng = np.random.default_rng(8)
    if table is None:
        table = synth.contact_table(rng)
    xs = np.arange(120) * 3.8
    long_chain = np.stack([xs, 2.0 * np.sin(xs / 7.0), 2.0 * np.cos(xs / 9.0)], axis=1)
    a = Molecule.from_beads(rng.integers(0, 20, 120), long_chain + np.array([10.0, 30.0, 30.0]))
    b = Molecule.from_beads(rng.integers(0, 20, 30),
                            synth.compact_chain(rng, 30) + np.array([30.0, 10.0, 45.0]))
    return System([a, b], 60.0, table)


def test_flags_match_the_bound(built_lib):
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import Engine
    w = synth.batch64(4, n_systems=16)
    systems = list(w.systems) + [_tight_box(w.systems[0].table)]  # one residue table
    with Engine(systems, 2, w.params) as eng:
        flags = eng.fold_flags()
    for s, f in zip(systems, flags):
        want, dist = _host_flag(s)
        if dist > 1e-3 * s.box:  # not on the edge of the bound
            assert f == want
    assert flags[-1] == 0
    assert flags[:-1].sum() > 0


def test_centre_far_outside_turns_the_fold_off(built_lib):
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import Engine
    w = synth.crowded(5)
    s = w.systems[0]
    with Engine([s], 1, w.params) as eng:
        assert eng.fold_flags()[0] == 1
        pos, rel, cen, quat = [a.copy() for a in s.state()]
        ms, _, _ = s.topology()
        shift = np.float32(3.0 * s.box)
        pos[ms[5]:ms[6], 0] += shift
        cen[5, 0] += shift
        eng.upload_state(pos, rel, cen, quat)
        assert eng.fold_flags()[0] == 0
        eng.upload_state(*s.state())
        assert eng.fold_flags()[0] == 1


def test_tight_box_trajectory_vs_oracle(built_lib):
    """The unfolded path where folding would be wrong."""
    from test_gpu_parity import _run_sweep_vs_oracle
    from remcdockingsimulator_b200 import synth
    s = _tight_box()
    R = 3
    w = synth.Workload("tight", [s], [R], [synth.geometric_ladder(300.0, 500.0, R)], 1.0, 0.2,
                       synth.benchmark_params(), 2000, 1000)
    _run_sweep_vs_oracle(w, R, 2000, seed=17)


def test_folded_batch_vs_oracle(built_lib):
    """The folded path on systems with chains and crowders, move for move."""
    from test_gpu_parity import _run_sweep_vs_oracle
    from remcdockingsimulator_b200 import synth
    w = synth.batch64(6, n_systems=3)
    for k in range(3):
        sub = synth.Workload("sub", [w.systems[k]], [2], [w.ladders[k][:2]], w.translate_step,
                             w.rotate_step, w.params, 800, 1000)
        _run_sweep_vs_oracle(sub, 2, 800, seed=100 + k)
