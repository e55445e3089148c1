"""The fluctuation estimate of d<B>/dlambda against a finite difference of <B>.

Config 0 (two chains of 76 and 24 residues, 100 A box, 20 replicas over
290-450 K) in 48 independent copies, each with its own replica exchange, run
by REMC at lambda - delta, lambda and lambda + delta with the same Philox
key. At config 0's own lambda (0.16) the chains stay bound at every
temperature of the ladder (<B> > 0.998), so the derivative is checked at
lambda = 0.07, where <B> falls from about 0.9 to 0.3 over the ladder. At lambda the driver's estimator (remc.SensitivitySums: the covariance
term -beta(<BX> - <B><X>) plus the bound threshold's term) gives d<B>/dlambda
per temperature; the runs at lambda +- delta give (<B>_+ - <B>_-) / 2 delta.
Both are averaged over the copies, and their statistical errors come from the
spread over the copies (the copies are independent). The test requires
agreement within 4 combined standard errors at every temperature whose <B>
is neither 0 nor 1, and that at least one such temperature exists.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COPIES = 48
BURN, STEPS, EVERY, BLOCK = 30000, 90000, 100, 1000


def _run(w, lam, seed, estimator):
    """Per copy: <B> per temperature, and (estimator) SensitivitySums."""
    from remcdockingsimulator_b200 import remc
    from remcdockingsimulator_b200.engine import Engine, make_params
    p = w.params
    q = make_params(lambda_=lam, e0=p.e0, debye_length=p.debye_length,
                    crowder_mode=p.crowder_mode, crowder_cutoff=p.crowder_cutoff,
                    crowder_eps=p.crowder_eps)
    s = w.systems[0]
    R = w.n_replicas[0]
    thr = float(remc.BOUND_ENERGY)
    nb = np.zeros((COPIES, R))
    ns = np.zeros((COPIES, R))
    sums = [remc.SensitivitySums(R) for _ in range(COPIES)]
    with Engine([s] * COPIES, [R] * COPIES, q) as eng:
        # the reference's step ladder (translations 0.5-5 A, rotations
        # 0.1-0.5 rad over the temperatures, main.cpp:1161-1178): the moves
        # leave the canonical distribution alone and the hot replicas travel
        ts, rs = remc.reference_step_ladder(R)
        eng.set_replica_params([w.ladders[0]] * COPIES, np.tile(ts, COPIES), np.tile(rs, COPIES))
        eng.energy_full()
        step = 0
        rnd = 0
        while step < BURN + STEPS:
            for _ in range(BLOCK // EVERY):
                eng.sweep(EVERY, seed, step)
                step += EVERY
                if step > BURN:
                    e = eng.energies().reshape(COPIES, R)
                    tmap = eng.temperature_map().reshape(COPIES, R)
                    X = eng.dE_dlambda().reshape(COPIES, R) if estimator else None
                    for c in range(COPIES):
                        np.add.at(nb[c], tmap[c], (e[c] < thr).astype(float))
                        np.add.at(ns[c], tmap[c], 1.0)
                        if estimator:
                            sums[c].add(tmap[c], e[c], X[c], 1.0)
            eng.exchange(seed, rnd, rnd & 1)
            rnd += 1
    return nb / ns, sums


def test_sensitivity_matches_finite_difference(built_lib):
    from remcdockingsimulator_b200 import remc, synth
    w = synth.two_chain(0)
    lam = 0.07
    delta = 0.05 * lam
    seed = 97
    B0, sums = _run(w, lam, seed, True)
    Bp, _ = _run(w, lam + delta, seed, False)
    Bm, _ = _run(w, lam - delta, seed, False)
    lam_p, lam_m = float(np.float32(lam + delta)), float(np.float32(lam - delta))
    fd = (Bp - Bm) / (lam_p - lam_m)                      # [copy, temperature]
    est = np.array([[row[6] for row in remc.sensitivity_estimates(w.ladders[0], sm.sums)]
                    for sm in sums])                      # [copy, temperature]
    mb = B0.mean(axis=0)
    informative = np.flatnonzero((mb > 0.05) & (mb < 0.95))
    assert informative.size > 0, mb
    se = lambda a: a.std(axis=0, ddof=1) / np.sqrt(COPIES)  # noqa: E731
    fd_m, fd_se = fd.mean(axis=0), se(fd)
    est_m, est_se = est.mean(axis=0), se(est)
    for t in informative:
        tol = 4.0 * np.hypot(fd_se[t], est_se[t])
        assert abs(fd_m[t] - est_m[t]) <= tol, (t, w.ladders[0][t], mb[t], fd_m[t], fd_se[t],
                                                est_m[t], est_se[t])
    # the estimate resolves a non-zero derivative somewhere
    assert np.max(np.abs(est_m[informative]) / est_se[informative]) > 4.0
