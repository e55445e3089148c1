"""CPU tests of the host driver: config grammar, flag overrides, placement
arithmetic, sampling-interval fit."""
import os

import numpy as np
import pytest


def _write_inputs(tmp, table):
    from remcdockingsimulator_b200.model import write_pdb_ca
    os.makedirs(os.path.join(tmp, "pdb"), exist_ok=True)
    rng = np.random.default_rng(0)
    a = rng.normal(size=(5, 3)).astype(np.float32) * 4
    write_pdb_ca(os.path.join(tmp, "pdb", "a.pdb"), [0, 1, 2, 3, 4], a, table)
    write_pdb_ca(os.path.join(tmp, "pdb", "c.pdb"), [0], np.zeros((1, 3), np.float32), table)
    cfg = os.path.join(tmp, "config")
    with open(cfg, "w") as fh:
        fh.write("# comment\nmcsteps 1000\nresteps 4\nreplicas 6\nsamplefrequency 70\n"
                 "sampleafter 0\nboundry 80\ntemperaturemax 300\ntemperaturemin 400\n"
                 "prefix test\ntemperaturetop 5\nthreads 99\nfiles\n"
                 "t(1.0,2.0,3.0) r(0,0,1,0.5) %s/pdb/a.pdb\n"
                 "p(10,20,30) r(1,1,0,-1) %s/pdb/a.pdb\n"
                 "garbage line\ncrowders\np(40,40,40) r(0,0,1,0.1) %s/pdb/c.pdb\n"
                 % (tmp, tmp, tmp))
    return cfg


def test_config_grammar_and_overrides(tmp_path, built_lib):
    from remcdockingsimulator_b200 import remc
    from remcdockingsimulator_b200.model import AminoAcidTable
    table = AminoAcidTable.synthetic()
    cfg = _write_inputs(str(tmp_path), table)
    a = remc.parse_cli(["-f", cfg, "-r", "8"])
    msgs = []
    mols = remc.load_config(a, table, log=msgs.append)
    assert a.mcsteps == 1000 and a.resteps == 4 and a.sample_frequency == 70
    assert a.prefix == "test_repulsive"
    assert (a.tmin, a.tmax) == (300.0, 400.0)  # swapped as the reference does
    assert a.threads == a.replicas  # capped at the replica count
    assert a.noncrowders == 2 and len(mols) == 3 and mols[2].crowder
    assert any("Failed to parse line" in m for m in msgs)
    remc.parse_cli(["-f", cfg, "-r", "8"], a)  # second pass
    assert a.replicas == 8
    # 't' translates (centre moves by the vector), 'p' places the centre
    m0 = mols[0]
    base = __import__("remcdockingsimulator_b200.model", fromlist=["Molecule"]).Molecule.from_pdb(
        os.path.join(str(tmp_path), "pdb", "a.pdb"), table)
    assert np.allclose(m0.centre, base.centre + np.float32([1, 2, 3]), atol=1e-5)
    assert np.array_equal(mols[1].centre, np.float32([10, 20, 30]))
    assert np.array_equal(mols[1].quat, [1.0, 0.0, 0.0, 0.0])  # angle -1: no rotation
    assert not np.array_equal(m0.quat, [1.0, 0.0, 0.0, 0.0])


def test_sample_frequency_fit(built_lib):
    from remcdockingsimulator_b200 import remc
    a = remc.Args(mcsteps=1000, resteps=4, sample_frequency=70)
    assert remc.adjusted_sample_frequency(a, log=lambda *_: None) == 125
    a = remc.Args(mcsteps=1000, resteps=4, sample_frequency=400)
    assert remc.adjusted_sample_frequency(a, log=lambda *_: None) == 250
    a = remc.Args(mcsteps=1000, resteps=4, sample_frequency=50)
    assert remc.adjusted_sample_frequency(a, log=lambda *_: None) == 50


def test_cli_flags(built_lib):
    from remcdockingsimulator_b200 import remc
    a = remc.parse_cli(["-m", "200", "-e", "2", "-t0", "280", "-t1", "310", "-b", "90.5",
                        "-bx", "64", "-z", "ck", "--seed", "7", "--unknown"])
    assert (a.mcsteps, a.resteps, a.tmin, a.tmax, a.bound, a.resume, a.seed) == \
        (200, 2, 280.0, 310.0, 90.5, "ck", 7)
    with pytest.raises(remc.ArgError):
        remc.parse_cli(["-m"])


def test_pdb_reader_repeats_last_bead_after_final_newline(tmp_path, built_lib):
    from remcdockingsimulator_b200.model import AminoAcidTable, read_pdb_ca
    table = AminoAcidTable.synthetic()
    p = tmp_path / "x.pdb"
    p.write_text("ATOM      1  CA  ALA A   1       1.000   2.000   3.000  1.00  1.00\n"
                 "ATOM      2  CA  GLY A   2       4.000   5.000   6.000  1.00  1.00\n")
    types, xyz = read_pdb_ca(str(p), table)
    assert len(types) == 3 and np.array_equal(xyz[1], xyz[2])  # Molecule.cpp:456-459
    p.write_text("ATOM      1  CA  ALA A   1       1.000   2.000   3.000  1.00  1.00\nEND\n")
    types, xyz = read_pdb_ca(str(p), table)
    assert len(types) == 1


def test_sensitivity_estimator(built_lib):
    """The fluctuation formula on synthetic samples: B = 1{X < 0} with X
    Gaussian; -beta(<BX> - <B><X>) = beta sigma phi(0) for zero-mean X."""
    from remcdockingsimulator_b200 import remc
    rng = np.random.default_rng(0)
    X = rng.normal(0.0, 2.0, size=200000)
    B = (X < 0).astype(float)
    sums = np.array([[len(X), B.sum(), X.sum(), (B * X).sum()]])
    (T, n, mb, mx, cov, surf, d), = remc.sensitivity_estimates(np.array([300.0]), sums)
    beta = 4184.0 / (8.314472 * 300.0)
    assert abs(mb - 0.5) < 0.01
    assert abs(d - beta * 2.0 / np.sqrt(2 * np.pi)) < 0.02 * beta
    assert surf == 0.0 and d == cov


def test_sensitivity_threshold_term(built_lib):
    """The threshold term <dB/dlambda> = -p(thr) <c X | E_nc = thr>, by the
    Gaussian kernel: energies N(mu, s^2), so the kernel estimate converges to
    the density of N(mu, s^2 + h^2) at the threshold; X = dE/dlambda a
    constant; c = 2 (crowders present)."""
    from remcdockingsimulator_b200 import remc
    rng = np.random.default_rng(1)
    mu, sd, h, x0 = -1.5, 0.8, 0.25, -7.0
    E = rng.normal(mu, sd, size=400000)
    acc = remc.SensitivitySums(1, bandwidth=h)
    acc.add(np.zeros(E.size, np.int64), E, np.full(E.size, x0), c=2.0)
    (T, n, mb, mx, cov, surf, d), = remc.sensitivity_estimates(np.array([300.0]), acc.sums)
    thr = float(remc.BOUND_ENERGY)
    s2 = sd * sd + h * h
    dens = np.exp(-0.5 * (thr - mu) ** 2 / s2) / np.sqrt(2 * np.pi * s2)
    assert n == E.size and abs(mb - np.mean(E < thr)) < 1e-12
    assert abs(cov) < 1e-9  # X does not fluctuate
    assert abs(surf - (-dens * 2.0 * x0)) < 0.01 * abs(dens * 2.0 * x0)
    assert abs(d - (cov + surf)) < 1e-12
