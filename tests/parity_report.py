"""Per-configuration parity report: the GPU engine against the FP64 oracle on
each benchmark configuration, in the spirit of the reference's check mode,
which prints CPU, GPU and error per structure (simulation engine/src/
main.cpp:1652-1707).

  python tests/parity_report.py [--configs 0,1,2,3,4] [--json FILE]

Configurations (built by remcdockingsimulator_b200.synth as bench.py builds
them; each handle under the schedule remc_autotune picks, as in the bench):
  0 two_chain  76 + 24 residues, 100 A box, 20 replicas
  1 crowded    config 0 + 400 crowders (R = 12 A, r^-12 walls), 32 replicas
  2 batch64    64 systems, 1024 replicas
  3 adjoint    4096 snapshots of config 1
  4 assembly   60 x 150 residues + 2000 crowders, 32 replicas

For configs 0, 1, 2 and 4 it reports
  E     max |E_gpu - E_64| / |E_64| of the full energy: every system at the
        start, and every followed replica after the run;
  dE    every accepted step of the sweep kernel on the followed replicas,
        one step per launch so that each step's dE_gpu is the change of the
        running energy, against the oracle's FP64 dE of the same move:
        max |dE_gpu - dE_64| / max(|dE_64|, S), S = the sum of the magnitudes
        of the moved molecule's pair terms at its old and new position (dE is
        a difference of two such sums and is ill-conditioned when it is far
        smaller than S); the largest absolute error; and the largest plain
        relative error over steps with |dE_64| >= 0.01 S;
  traj  whether coordinates, rotations and decisions stayed identical.
For config 3 it reports the adjoint against FP64 central differences of the
oracle's energy: forces (h = 1e-4 A on each coordinate of the 30 beads with
the largest force and 10 others), dE/dlambda (lambda +- 1%: the energy is
linear in lambda), dE/dXi (Xi +- 1e-4 A) and dE/deps (the 10 diagonal and 20
largest off-diagonal entries, eps +- 1e-3: linear), and the energy of 64
snapshots against the oracle's.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _rel(a, b, floor=1e-3):
    return abs(a - b) / max(abs(b), floor)


def sweep_report(w, followed, n_steps, seed):
    from oracle import bindings as ob
    from remcdockingsimulator_b200.engine import Engine
    out = {"workload": w.name, "systems": len(w.systems), "replicas": w.n_inst,
           "steps": n_steps}
    oracles = {}

    def o_of(si):
        if si not in oracles:
            oracles[si] = ob.FP64Oracle(w.systems[si], w.params)
        return oracles[si]

    with Engine(w.systems, w.n_replicas, w.params) as eng:
        eng.set_replica_params(w.ladders, np.full(len(w.systems), w.translate_step, np.float32),
                               np.full(len(w.systems), w.rotate_step))
        e0 = eng.energy_full()
        t, smem, _ = eng.autotune(probe_steps=min(256, n_steps))
        out["schedule"] = {"threads": int(t), "centres_in_shared_memory": bool(smem),
                           "ctas_per_replica": int(eng.schedule()[2]),
                           "beads_in_shared_memory": bool(eng.beads_in_shared_memory())}
        e_start = 0.0
        for si, s in enumerate(w.systems):
            e_start = max(e_start, _rel(e0[eng.inst_first[si]], o_of(si).energy(s.state()[0])))
        out["E_start_max_rel"] = e_start
        insts = [eng.inst_first[si] + k for si, k in followed]
        traj = np.zeros((n_steps, len(insts)))
        prev = e0[insts]
        for step in range(n_steps):
            eng.sweep(1, seed, step)
            e = eng.energies()[insts]
            traj[step] = e - prev
            prev = e
        st = eng.download_state()
        e_full = eng.energy_full()
        slices = eng.instance_slices()
    worst_c = worst_abs = worst_raw = 0.0
    n_acc = 0
    e_end = 0.0
    identical = True
    ts, rs = float(np.float32(w.translate_step)), float(w.rotate_step)
    for c, (si, k) in enumerate(followed):
        s = w.systems[si]
        o = o_of(si)
        ms = s.topology()[0]
        inst = insts[c]
        state = s.state()
        E = float(e0[inst])
        T = float(w.ladders[si][k])
        for step in range(n_steps):
            new, E, flags, mol, dE, _ = o.mc_run(state, T, ts, rs, seed, step, k, si, 1, E)
            if flags[0]:
                m = int(mol[0])
                a, b = ms[m], ms[m + 1]
                S = (o.energy_molecule_abs(state[0], m, new[0][a:b]) +
                     o.energy_molecule_abs(state[0], m, state[0][a:b]))
                d64, dg = float(dE[0]), float(traj[step, c])
                err = abs(dg - d64)
                worst_c = max(worst_c, err / max(abs(d64), S, 1e-12))
                worst_abs = max(worst_abs, err)
                if abs(d64) >= 0.01 * S:
                    worst_raw = max(worst_raw, err / abs(d64))
                n_acc += 1
            state = new
        bs, msl = slices[inst]
        identical &= bool(np.array_equal(st[0][bs], state[0]) and
                          np.array_equal(st[3][msl], state[3]))
        e_end = max(e_end, _rel(e_full[inst], o.energy(state[0])))
    out.update({"followed_replicas": len(followed), "accepted_steps": n_acc,
                "E_end_max_rel": e_end, "dE_max_conditioned": worst_c, "dE_max_abs": worst_abs,
                "dE_max_rel_well_conditioned": worst_raw, "trajectories_identical": identical})
    return out


def adjoint_report(n_snap=4096, seed=7):
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import Engine, make_params
    w = synth.crowded(seed)
    s = w.systems[0]
    p = w.params
    with Engine([s], [n_snap], p) as eng:
        eng.set_replica_params([np.linspace(290, 480, n_snap).astype(np.float32)],
                               [w.translate_step], [w.rotate_step])
        eng.energy_full()
        eng.sweep(200, seed + 9, 0)
        st = eng.download_state()
        full = eng.energy_full()
        adj = eng.adjoint()
        sl = eng.instance_slices()
    o = ob.FP64Oracle(s, p)
    e_err = 0.0
    for k in np.linspace(0, n_snap - 1, 64).astype(int):
        e_err = max(e_err, _rel(full[k], o.energy(st[0][sl[k][0]])),
                    _rel(adj["energy"][k], o.energy(st[0][sl[k][0]])))
    rng = np.random.default_rng(3)
    f_err = f_el = dl_err = dx_err = de_err = 0.0
    for k in (0, n_snap - 1):
        bs = sl[k][0]
        pos = st[0][bs].copy()
        fg = adj["forces"][bs].astype(np.float64)
        mag = np.abs(fg).max(axis=1)
        beads = list(np.argsort(-mag)[:30]) + list(rng.choice(len(pos), 10, replace=False))
        fd, fgs = [], []
        for bead in beads:
            for c in range(3):
                pp, pm = pos.copy(), pos.copy()
                pp[bead, c] = np.float32(pos[bead, c] + 1e-4)
                pm[bead, c] = np.float32(pos[bead, c] - 1e-4)
                h2 = float(pp[bead, c]) - float(pm[bead, c])
                fd.append(-(o.energy(pp) - o.energy(pm)) / h2)
                fgs.append(fg[bead, c])
        fd, fgs = np.array(fd), np.array(fgs)
        f_err = max(f_err, np.linalg.norm(fgs - fd) / np.linalg.norm(fd))
        big = np.abs(fd) > 0.01 * np.abs(fd).max()
        f_el = max(f_el, float(np.max(np.abs(fgs[big] - fd[big]) / np.abs(fd[big]))))
        # dE/dlambda: lambda -+ 1%
        lam = float(p.lambda_)
        e_l = []
        for l in (lam * 1.01, lam * 0.99):
            q = make_params(lambda_=l, e0=p.e0, debye_length=p.debye_length,
                            crowder_mode=p.crowder_mode, crowder_cutoff=p.crowder_cutoff,
                            crowder_eps=p.crowder_eps)
            e_l.append(ob.FP64Oracle(s, q).energy(pos))
        lp, lm = float(np.float32(lam * 1.01)), float(np.float32(lam * 0.99))
        dl_fd = (e_l[0] - e_l[1]) / (lp - lm)
        dl_err = max(dl_err, _rel(adj["dE_dlambda"][k], dl_fd, 1e-9))
        # dE/dXi: Xi -+ 1e-4 A (the FP32 values actually used)
        xi = float(p.debye_length)
        e_x = []
        xs = [float(np.float32(xi + 1e-4)), float(np.float32(xi - 1e-4))]
        for x in xs:
            q = make_params(lambda_=p.lambda_, e0=p.e0, debye_length=x,
                            crowder_mode=p.crowder_mode, crowder_cutoff=p.crowder_cutoff,
                            crowder_eps=p.crowder_eps)
            e_x.append(ob.FP64Oracle(s, q).energy(pos))
        dx_fd = (e_x[0] - e_x[1]) / (xs[0] - xs[1])
        dx_err = max(dx_err, _rel(adj["dE_dxi"][k], dx_fd, 1e-9))
        # dE/deps_ab (symmetric entry): eps -+ 1e-3 in the oracle's FP32 table
        deg = adj["dE_deps"][k]
        off = [(a, b) for a in range(20) for b in range(a + 1, 20)]
        off.sort(key=lambda ab: -abs(deg[ab[0], ab[1]]))
        entries = [(a, a) for a in range(10)] + off[:20]
        for a, b in entries:
            base = o.eps.copy()
            v = float(o.eps[a * 32 + b])
            if abs(v) < 2e-3:
                continue
            vals = []
            ev = []
            for dv in (1e-3, -1e-3):
                nv = np.float32(v + dv)
                o.eps[a * 32 + b] = nv
                o.eps[b * 32 + a] = nv
                ev.append(o.energy(pos))
                vals.append(float(nv))
            o.eps[:] = base
            de_fd = (ev[0] - ev[1]) / (vals[0] - vals[1])
            de_err = max(de_err, _rel(deg[a, b], de_fd, 1e-6 * np.abs(deg).max()))
    return {"workload": "crowded snapshots", "snapshots": n_snap, "E_max_rel_64_snapshots": e_err,
            "forces_rel_l2": f_err, "forces_max_rel_elementwise": f_el,
            "dE_dlambda_rel": dl_err, "dE_dxi_rel": dx_err, "dE_deps_max_rel": de_err}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--configs", default="0,1,2,3,4")
    ap.add_argument("--json", default="")
    args = ap.parse_args()
    import torch
    torch.cuda.set_device(0)
    from remcdockingsimulator_b200 import synth
    report = {}
    for c in [int(x) for x in args.configs.split(",")]:
        t0 = time.time()
        if c == 0:
            w = synth.two_chain(0)
            r = sweep_report(w, [(0, k) for k in range(20)], 1000, 501)
        elif c == 1:
            w = synth.crowded(0)
            r = sweep_report(w, [(0, k) for k in range(0, 32, 4)], 1000, 502)
        elif c == 2:
            w = synth.batch64(0)
            n_b = np.array([s.n_beads for s in w.systems])
            n_cr = np.array([sum(1 for m in s.molecules if m.crowder) for s in w.systems])
            picks = []
            for si in (int(n_b.argmin()), int(n_b.argmax()), int(n_cr.argmax()),
                       int(n_cr.argmin()), 17, 42):
                if si not in picks:
                    picks.append(si)
            r = sweep_report(w, [(si, k) for si in picks for k in (0, 15)], 1000, 503)
        elif c == 3:
            r = adjoint_report()
        elif c == 4:
            w = synth.assembly(0)
            r = sweep_report(w, [(0, 0), (0, 31)], 300, 504)
        else:
            continue
        r["seconds"] = round(time.time() - t0, 1)
        report["config%d" % c] = r
        print(json.dumps({"config": c, **r}), flush=True)
    if args.json:
        with open(args.json, "w") as fh:
            json.dump(report, fh, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
