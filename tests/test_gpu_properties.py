"""Randomised property tests of the GPU engine (hypothesis, derandomised so
that every run draws the same examples): invariance of the full energy under
a global translation and under moving a molecule by whole box lengths, the
single-move energy difference equal to the difference of full energies, a
rejected step leaving the state bit-identical, and an instance's energy
independent of what else is batched with it."""
import numpy as np
import pytest
from hypothesis import given, settings
from hypothesis import strategies as st

pytestmark = pytest.mark.gpu
E_RTOL = 1e-5
PROPS = settings(max_examples=8, deadline=None, derandomize=True)


def _system(which, seed):
    from remcdockingsimulator_b200 import synth
    w = synth.crowded(seed) if which == "crowded" else synth.two_chain(seed)
    return w.systems[0], w.params


def _energy(s, params, state=None):
    from remcdockingsimulator_b200.engine import Engine
    with Engine([s], 1, params) as eng:
        if state is not None:
            eng.upload_state(*state)
        return float(eng.energy_full()[0])


def _close(a, b, scale):
    # relative to the energy's size, with a 1e-6 kcal/mol floor for systems
    # whose energy is near zero (moving coordinates rounds them in FP32)
    return abs(a - b) <= E_RTOL * scale + 1e-6


@PROPS
@given(which=st.sampled_from(["crowded", "two_chain"]),
       t=st.tuples(*[st.floats(-50.0, 50.0) for _ in range(3)]))
def test_energy_invariant_under_global_translation(built_lib, which, t):
    s, params = _system(which, 3)
    pos, rel, cen, quat = s.state()
    v = np.array(t, np.float32)
    e0 = _energy(s, params)
    e1 = _energy(s, params, ((pos + v).astype(np.float32), rel, (cen + v).astype(np.float32), quat))
    assert _close(e0, e1, abs(e0)), (e0, e1)


@PROPS
@given(which=st.sampled_from(["crowded", "two_chain"]),
       mol=st.integers(0, 400), k=st.tuples(*[st.integers(-2, 2) for _ in range(3)]))
def test_energy_invariant_under_box_shifts(built_lib, which, mol, k):
    s, params = _system(which, 4)
    pos, rel, cen, quat = [a.copy() for a in s.state()]
    mol = mol % s.n_mol
    ms, _, _ = s.topology()
    shift = (np.array(k, np.float32) * np.float32(s.box)).astype(np.float32)
    e0 = _energy(s, params)
    pos[ms[mol]:ms[mol + 1]] += shift
    cen[mol] += shift
    e1 = _energy(s, params, (pos, rel, cen, quat))
    assert _close(e0, e1, abs(e0)), (e0, e1)


@PROPS
@given(mol=st.integers(0, 401), d=st.tuples(*[st.floats(-6.0, 6.0) for _ in range(3)]))
def test_delta_energy_is_difference_of_full_energies(built_lib, mol, d):
    from remcdockingsimulator_b200.engine import Engine
    s, params = _system("crowded", 5)
    pos, rel, cen, quat = [a.copy() for a in s.state()]
    mol = mol % s.n_mol
    ms, _, _ = s.topology()
    v = np.array(d, np.float32)
    new = (pos[ms[mol]:ms[mol + 1]] + v).astype(np.float32)
    with Engine([s], 1, params) as eng:
        e0 = float(eng.energy_full()[0])
        de = eng.delta_energy(0, mol, new)
        pos[ms[mol]:ms[mol + 1]] = new
        cen[mol] = (cen[mol] + v).astype(np.float32)
        eng.upload_state(pos, rel, cen, quat)
        e1 = float(eng.energy_full()[0])
    scale = abs(e0) + abs(e1)
    assert _close(de, e1 - e0, scale), (de, e1 - e0)


@PROPS
@given(seed=st.integers(0, 2**31 - 1))
def test_rejected_step_leaves_state_unchanged(built_lib, seed):
    from remcdockingsimulator_b200.engine import Engine
    s, params = _system("crowded", 6)
    with Engine([s], 1, params) as eng:
        # a low temperature, so that most moves that raise the energy are rejected
        eng.set_replica_params([np.array([5.0], np.float32)], [np.float32(3.0)], [0.5])
        eng.energy_full()
        found = False
        for step in range(64):
            before = eng.download_state()
            e_before = eng.energies()[0]
            eng.reset_counters()
            eng.sweep(1, seed, step)
            if eng.counters()[2][0] == 1:  # rejected
                after = eng.download_state()
                for a, b in zip(before, after):
                    assert np.array_equal(a, b)
                assert eng.energies()[0] == e_before
                found = True
                break
        assert found, "no rejected step in 64 tries"


def test_energy_independent_of_batch_companions(built_lib):
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import Engine
    w = synth.WORKLOADS["batch64"](2)
    s = w.systems[0]
    alone = _energy(s, w.params)
    with Engine([w.systems[3], s, w.systems[7]], [2, 3, 1], w.params) as eng:
        e = eng.energy_full()
    # instances 2..4 hold system s; per-item partials are summed in a fixed order
    assert np.all(e[2:5] == alone), (e[2:5], alone)
