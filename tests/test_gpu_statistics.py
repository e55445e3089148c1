"""Statistical parity with the reference's own engine under independent
random streams: the GPU sweep (Philox) and the reference's Replica::MCSearch
(compiled from its sources, its own MT19937 generators) start from the same
two-chain conformation in a 50 A box and run 3000 steps at 300 K and 400 K.
Energies sampled at steps 1000, 1500, ..., 3000 over independent replicas must
come from the same distribution (two-sample Kolmogorov-Smirnov, p > 1e-3 per
temperature) and the acceptance rates must agree within 0.03.

This complements the bitwise tests (same stream on both sides): it checks
the dynamics in distribution, with each side drawing its own numbers."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TEMPS = (300.0, 400.0)
STEPS, CHUNK, FIRST_SAMPLE = 3000, 500, 1000
N_GPU, N_REF = 128, 24
TSTEP, RSTEP = 0.5, 0.2


def _system():
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.model import System
    s0 = synth.two_chain(21).systems[0]
    return System([m.copy() for m in s0.molecules], 50.0, s0.table)


def _gpu_samples(s):
    from remcdockingsimulator_b200.engine import Engine, make_params
    R = N_GPU * len(TEMPS)
    ladder = np.repeat(np.array(TEMPS, np.float32), N_GPU)
    samples = {T: [] for T in TEMPS}
    with Engine([s], R, make_params()) as eng:  # the reference's constants
        eng.set_replica_params([ladder], np.full(R, TSTEP, np.float32), np.full(R, RSTEP))
        eng.energy_full()
        for c in range(STEPS // CHUNK):
            eng.sweep(CHUNK, 424242, c * CHUNK)
            if (c + 1) * CHUNK >= FIRST_SAMPLE:
                e = eng.energies()
                for t, T in enumerate(TEMPS):
                    samples[T].extend(e[t * N_GPU:(t + 1) * N_GPU].tolist())
        acc, accA, rej = eng.counters()
    rates = {}
    for t, T in enumerate(TEMPS):
        sl = slice(t * N_GPU, (t + 1) * N_GPU)
        ok = acc[sl].sum() + accA[sl].sum()
        rates[T] = ok / float(ok + rej[sl].sum())
    return samples, rates


def _reference_samples(s):
    from oracle import bindings as ob
    reps = {}
    for T in TEMPS:
        reps[T] = []
        for k in range(N_REF):
            r = ob.ReferenceReplica(s, temperature=T)
            r.set_steps(TSTEP, RSTEP)
            r.seed(9000 + 131 * k + int(T))
            reps[T].append(r)
    allr = [r for T in TEMPS for r in reps[T]]
    samples = {T: [] for T in TEMPS}
    for c in range(STEPS // CHUNK):
        ob.run_reference_mcsearch(allr, 8, CHUNK)
        if (c + 1) * CHUNK >= FIRST_SAMPLE:
            for T in TEMPS:
                samples[T].extend(r.potential for r in reps[T])
    rates = {}
    for T in TEMPS:
        cnt = np.array([r.counters() for r in reps[T]])
        rates[T] = (cnt[:, 0].sum() + cnt[:, 1].sum()) / float(cnt.sum())
    for r in allr:
        r.close()
    return samples, rates


def test_energy_distributions_and_acceptance_match_reference(built_lib):
    from scipy import stats
    from oracle import bindings as ob
    if not ob.reference_available():
        pytest.skip("reference harness not built")
    s = _system()
    g_samples, g_rates = _gpu_samples(s)
    r_samples, r_rates = _reference_samples(s)
    for T in TEMPS:
        res = stats.ks_2samp(g_samples[T], r_samples[T])
        assert res.pvalue > 1e-3, (T, res, np.mean(g_samples[T]), np.mean(r_samples[T]))
        assert abs(g_rates[T] - r_rates[T]) < 0.03, (T, g_rates[T], r_rates[T])
    # the two temperatures are distinguishable (the test has power)
    assert g_rates[400.0] > g_rates[300.0]
