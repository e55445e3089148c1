"""CPU tests: the FP64 oracle pinned against the reference's golden data and
its own compiled CPU engine; host-side model and file formats."""
import math
import os

import numpy as np
import pytest

from conftest import golden_system


# ---------------------------------------------------------------- Philox
def test_philox_known_answers(oracle_built):
    """Philox4x32-10 known-answer vectors published with Random123."""
    from oracle import bindings as ob
    assert ob.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert ob.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                             0x6D5451FD]
    assert ob.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                     [0xA4093822, 0x299F31D0]) == [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_step_uniforms_layout(oracle_built):
    from oracle import bindings as ob
    u = ob.step_uniforms(0x1234_5678_9ABC, 7, 3, 2)
    x = ob.philox([7, 3, 2, 0], [0x56789ABC, 0x1234])
    y = ob.philox([7, 3, 2, 1], [0x56789ABC, 0x1234])
    assert np.allclose(u, [x[0] / 2**32, x[1] / 2**32, x[2] / 2**32, x[3] / 2**32,
                           y[0] / 2**32, y[1] / 2**32], rtol=0, atol=0)


# ---------------------------------------------------------------- golden
def test_oracle_vs_golden_reference_energies(golden, golden_table, oracle_built, built_lib):
    """The FP64 oracle reproduces the reference Replica::E() values on the 10
    golden structures (118.4 A box) to 1e-6 relative (structure 5, whose energy
    is ~1e-4 kcal/mol, to 1e-9 absolute)."""
    from oracle import bindings as ob
    from remcdockingsimulator_b200.engine import make_params
    p = make_params()
    for k, st in enumerate(golden["structures"]):
        s = golden_system(golden, golden_table, k)
        e = ob.FP64Oracle(s, p).energy(s.state()[0])
        ref = st["reference_E"]
        if abs(ref) > 1e-2:
            assert abs(e - ref) / abs(ref) < 1e-6, (k, e, ref)
        else:
            assert abs(e - ref) < 1e-9, (k, e, ref)


def test_oracle_vs_independent_implementation(golden, golden_table, oracle_built, built_lib):
    """Loose pin against the independent implementation shipped with the
    reference (ref_ene / pairs_N.dat): ~0.1-1% on totals."""
    from oracle import bindings as ob
    from remcdockingsimulator_b200.engine import make_params
    p = make_params()
    for k, st in enumerate(golden["structures"]):
        s = golden_system(golden, golden_table, k)
        e = ob.FP64Oracle(s, p).energy(s.state()[0])
        ind = st["independent_total"]
        assert abs(st["pair_file_sums"]["total"] - ind) < 5e-3 * max(1.0, abs(ind))
        if abs(ind) > 1.0:
            assert abs(e - ind) / abs(ind) < 1.5e-2, (k, e, ind)
        old = st["energy_txt_total"]
        if abs(old) > 1.0:
            assert abs(e - old) / abs(old) < 1.5e-2, (k, e, old)


def test_golden_structure_shapes(golden):
    for st in golden["structures"]:
        assert [len(c["types"]) for c in st["chains"]] == [24, 76]


# ---------------------------------------------------------------- reference engine
from oracle.build import reference_src  # noqa: E402

ref_needed = pytest.mark.skipif(
    not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref",
                                    "libremcref.so")) and
    not os.path.isdir(reference_src()),
    reason="reference harness not built here")


@ref_needed
def test_reference_harness_reproduces_golden(golden, golden_table, built_lib):
    from oracle import bindings as ob
    for k in (0, 2, 7):
        s = golden_system(golden, golden_table, k)
        r = ob.ReferenceReplica(s)
        assert r.E() == pytest.approx(golden["structures"][k]["reference_E"], rel=1e-12, abs=1e-15)
        assert r.E_pair(0, 1) == pytest.approx(golden["structures"][k]["reference_E_pair"],
                                               rel=1e-6)
        r.close()


@ref_needed
@pytest.mark.parametrize("seed", [1, 99])
def test_oracle_mc_trajectory_bitwise_vs_reference(seed, built_lib):
    """The reference's own MCSearch, fed the shared Philox stream, and the
    oracle's move arithmetic give bit-identical coordinates and the same
    accept/reject decisions."""
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import make_params
    w = synth.two_chain(seed)
    s = w.systems[0]
    p = make_params()
    o = ob.FP64Oracle(s, p)
    r = ob.ReferenceReplica(s, temperature=310.0)
    r.set_steps(1.5, 0.3)
    n = 400
    u = np.stack([ob.step_uniforms(seed, t, 0, 0) for t in range(n)])
    fr, mr, er, under = r.mcsearch(u)
    assert under == 0
    st, E, fo, mo, dE, cnt = o.mc_run(s.state(), 310.0, 1.5, 0.3, seed, 0, 0, 0, n,
                                      o.energy(s.state()[0]), energy_mode=1)
    assert np.array_equal(mr, mo)
    # decisions agree except where the Metropolis margin is below the FP32 noise
    mism = np.flatnonzero((fr > 0) != (fo > 0))
    assert mism.size == 0, mism
    sr = r.state()
    for a, b in zip(sr, st):
        assert np.array_equal(a, b)
    assert E == pytest.approx(er[-1], rel=1e-6, abs=1e-9)


@ref_needed
def test_reference_random_vectors_mapping(built_lib):
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    import ctypes as C
    s = synth.two_chain(0).systems[0]
    r = ob.ReferenceReplica(s)
    u3 = np.array([0.9, 0.2, 0.6])
    vf = np.zeros(3, np.float32)
    vd = np.zeros(3)
    ob.ref_lib().ref_random_vectors(r.h, u3.ctypes.data_as(C.POINTER(C.c_double)),
                                    vf.ctypes.data_as(C.POINTER(C.c_float)),
                                    vd.ctypes.data_as(C.POINTER(C.c_double)))
    raw = np.array([0.9 - 0.5, 0.5 - 0.2, 0.6 - 0.5])
    assert np.allclose(vd, raw / np.linalg.norm(raw), rtol=0, atol=1e-15)
    assert np.allclose(vf, raw / np.linalg.norm(raw), rtol=1e-6)


# ---------------------------------------------------------------- oracle internals
def test_oracle_delta_matches_full_difference(oracle_built, built_lib):
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    w = synth.crowded(3)
    s = w.systems[0]
    o = ob.FP64Oracle(s, w.params)
    pos = s.state()[0].copy()
    e0 = o.energy(pos)
    ms = s.topology()[0]
    for m in (0, 1, 5, 300):
        new = pos[ms[m]:ms[m + 1]] + np.float32(0.7)
        d = o.energy_molecule(pos, m, new) - o.energy_molecule(pos, m, pos[ms[m]:ms[m + 1]])
        p2 = pos.copy()
        p2[ms[m]:ms[m + 1]] = new
        assert d == pytest.approx(o.energy(p2) - e0, rel=1e-9, abs=1e-9)


def test_oracle_exchange_round_semantics(oracle_built):
    from oracle import bindings as ob
    lad = np.array([300, 310, 320, 330, 340], np.float32)
    en = np.array([-5.0, -1.0, -3.0, 2.0, -10.0])
    tos = np.arange(5, dtype=np.int32)
    n, tos2, sot2, acc = ob.exchange_round(lad, en, tos, tos, 0, 42, 0, 0)
    # every accepted pair is a swap of neighbouring temperatures
    for t in range(0, 4, 2):
        a, b = t, t + 1
        if acc[t // 2]:
            assert tos2[a] == t + 1 and tos2[b] == t
    assert np.array_equal(np.sort(tos2), np.arange(5))
    assert np.array_equal(sot2[tos2], np.arange(5))
    # pair (3,4): E_3 - E_4 = 12 > 0 with T_3 < T_4 -> delta > 0 -> always accepted
    assert acc[1] == 1


def test_oracle_translation_invariance(oracle_built, built_lib):
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    w = synth.two_chain(5)
    s = w.systems[0]
    o = ob.FP64Oracle(s, w.params)
    pos = s.state()[0]
    e = o.energy(pos)
    shifted = (pos + np.float32(s.box)).astype(np.float32)  # one box image
    assert o.energy(shifted) == pytest.approx(e, rel=1e-5)


def test_mixed_crowder_species_topology(oracle_built):
    """Crowders with their own radii become species 20, 21, ... in order of
    first appearance, carrying those radii in the type tables."""
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    w = synth.crowded(3)
    s = w.systems[0]
    radii = (12.0, 9.0, 7.0)
    crowders = [m for m in s.molecules if m.crowder]
    for k, m in enumerate(crowders):
        m.radius = radii[k % 3]
    assert s.crowder_radii() == list(radii)
    _, _, types = s.topology()
    ncb = sum(m.n for m in s.molecules if not m.crowder)
    assert list(types[ncb:ncb + 6]) == [20, 21, 22, 20, 21, 22]
    assert list(s.type_tables()[2][20:23]) == list(radii)
    # in the r^-12 model the radii enter the energy
    e_mixed = ob.FP64Oracle(s, w.params).energy(s.state()[0])
    for m in crowders:
        m.radius = None
    e_one = ob.FP64Oracle(s, w.params).energy(s.state()[0])
    assert abs(e_mixed - e_one) > 1e-3 * abs(e_one)
