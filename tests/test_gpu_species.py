"""Crowders of several species (radii) in one system. The kernels then have
no single crowder table entry per system and take their mixed paths: the
full energy in both crowder models, the sweep's one-bead and chain loops,
and the adjoint's per-bead crowder lookups, each against the oracle. Also an
engine whose systems use different radii, mapped onto shared species types."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
E_RTOL = 1e-5


def _mixed(seed, radii=(12.0, 9.0, 7.0)):
    """The crowded workload with its crowders cycling through `radii` (all no
    larger than the 12 A they were placed with, so nothing overlaps)."""
    from remcdockingsimulator_b200 import synth
    w = synth.crowded(seed)
    k = 0
    for m in w.systems[0].molecules:
        if m.crowder:
            m.radius = radii[k % len(radii)]
            k += 1
    return w


def _energies(systems, params, R=2):
    from remcdockingsimulator_b200.engine import Engine
    with Engine(systems, R, params) as eng:
        return eng.energy_full()


@pytest.mark.parametrize("model", ["r12", "reference"])
def test_mixed_species_energy_vs_oracle(model, built_lib):
    from oracle import bindings as ob
    from remcdockingsimulator_b200.engine import make_params
    w = _mixed(4)
    s = w.systems[0]
    p = w.params if model == "r12" else make_params(lambda_=0.16)
    e = _energies([s], p)
    ref = ob.FP64Oracle(s, p).energy(s.state()[0])
    assert np.all(np.abs(e - ref) <= E_RTOL * max(abs(ref), 1e-3)), (e, ref)
    # one species for all: a different energy in the r^-12 model (the radii matter)
    if model == "r12":
        for m in s.molecules:
            m.radius = None
        assert abs(_energies([s], p)[0] - ref) > 1e-3 * abs(ref)


def test_mixed_species_sweep_vs_oracle(built_lib):
    from test_gpu_parity import _run_sweep_vs_oracle
    _run_sweep_vs_oracle(_mixed(5), 3, 1500, seed=41)


def test_mixed_species_adjoint_vs_oracle(built_lib):
    from test_gpu_adjoint import _check
    _check("crowded", 6, w=_mixed(6))


def test_systems_with_different_radii_share_species(built_lib):
    """Three copies of one system in one engine: all crowders 12 A, all 8 A,
    and both; every instance's energy equals its own system's oracle energy."""
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.model import System
    w = synth.crowded(7)
    a = w.systems[0]

    def clone(radius, radii=None):
        mols = [m.copy() for m in a.molecules]
        k = 0
        for m in mols:
            if m.crowder and radii:
                m.radius = radii[k % len(radii)]
                k += 1
        return System(mols, a.box, a.table, crowder_radius=radius,
                      translate_only_crowders=a.translate_only_crowders)

    systems = [clone(12.0), clone(8.0), clone(12.0, (8.0, 12.0))]
    e = _energies(systems, w.params, R=2)
    refs = [ob.FP64Oracle(s, w.params).energy(s.state()[0]) for s in systems]
    for k, ref in enumerate(refs):
        assert np.all(np.abs(e[2 * k:2 * k + 2] - ref) <= E_RTOL * max(abs(ref), 1e-3)), (k, e, ref)
    assert len({round(r, 3) for r in refs}) == 3  # the radii change the energy
