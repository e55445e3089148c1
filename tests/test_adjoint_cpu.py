"""CPU: the FP64 oracle's analytic adjoint against FP64 central finite
differences of its own energy (h = 1e-4 A for positions, 1e-5 for the
parameters). Systems avoid pairs near the 15 A crowder cutoff by using the
r^-12 crowder model without a cutoff."""
import ctypes as C

import numpy as np
import pytest


def _system(seed):
    from remcdockingsimulator_b200 import synth
    rng = np.random.default_rng(seed)
    table = synth.contact_table(rng)
    return synth.build_system(rng, table, [12, 9], 6, 8.0, 60.0), synth.benchmark_params()


def test_oracle_forces_match_central_differences(oracle_built, built_lib):
    from oracle import bindings as ob
    s, p = _system(3)
    o = ob.FP64Oracle(s, p)
    pos = s.state()[0].astype(np.float32)
    f, dl, dx, de = o.adjoint(pos)
    # FD in FP32 coordinates needs a step the FP32 grid can resolve; use the
    # largest-force beads and h = 1e-3 A around representable positions
    h = 1e-3
    idx = np.argsort(-np.abs(f).max(axis=1))[:6]
    for b in idx:
        for k in range(3):
            pp = pos.copy()
            pm = pos.copy()
            pp[b, k] = np.float32(pos[b, k] + h)
            pm[b, k] = np.float32(pos[b, k] - h)
            hh = (float(pp[b, k]) - float(pm[b, k])) / 2.0
            fd = -(o.energy(pp) - o.energy(pm)) / (2 * hh)
            assert abs(fd - f[b, k]) <= 2e-3 * max(abs(f[b, k]), 1e-2), (b, k, fd, f[b, k])


def test_oracle_parameter_derivatives_match_central_differences(oracle_built, built_lib):
    from oracle import bindings as ob
    s, p = _system(4)
    pos = s.state()[0].astype(np.float32)
    o = ob.FP64Oracle(s, p)
    f, dl, dx, de = o.adjoint(pos)
    # Debye length (parameter of the DH term, continuous)
    h = 1e-5 * float(p.debye_length)

    def e_with(**kw):
        import copy
        q = ob.params_from(p)
        for k, v in kw.items():
            setattr(q, k, v)
        o2 = ob.FP64Oracle(s, q)
        return o2.energy(pos)
    xp = float(np.float32(p.debye_length + h))
    xm = float(np.float32(p.debye_length - h))
    fd_xi = (e_with(debye_length=xp) - e_with(debye_length=xm)) / (xp - xm)
    assert abs(fd_xi - dx) <= 1e-3 * max(abs(dx), 1e-4), (fd_xi, dx)
    # eps_ab: perturb one symmetric table entry of the oracle directly
    a, b = 3, 7
    o_p = ob.FP64Oracle(s, p)
    o_m = ob.FP64Oracle(s, p)
    he = 1e-3
    for oo, sgn in ((o_p, 1), (o_m, -1)):
        e = oo.eps.reshape(32, 32)
        e[a, b] = np.float32(e[a, b] + sgn * he)
        e[b, a] = e[a, b]
    fd_e = (o_p.energy(pos) - o_m.energy(pos)) / (
        float(o_p.eps.reshape(32, 32)[a, b]) - float(o_m.eps.reshape(32, 32)[a, b]))
    assert abs(fd_e - de[a, b]) <= 1e-3 * max(abs(de[a, b]), 1e-6), (fd_e, de[a, b])
    # lambda: eps = lambda (M - e0) for every residue pair
    M = s.table.pairs.astype(np.float64)
    # dE/dlambda equals sum over unordered type pairs of dE/deps_ab (M_ab - e0)
    tot = 0.0
    for i in range(20):
        for j in range(i, 20):
            tot += de[i, j] * (float(M[i, j]) - float(p.e0))
    assert abs(tot - dl) <= 1e-9 * max(1.0, abs(dl)), (tot, dl)
