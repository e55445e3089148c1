"""Replica-exchange driver with the reference's config format, flags and
output files.

  python -m remcdockingsimulator_b200 -f <config> [-m mcsteps] [-e resteps] ...

Mirrors, on top of the batched GPU engine:
  loadArgsFromFile ... simulation engine/src/main.cpp:383-632 (config file)
  getArgs ............ main.cpp:193-381 (command-line overrides)
  REMCSimulation ..... main.cpp:1106-1567 (ladder, blocks, sampling files,
                       neighbour exchanges, REsteps - 1 exchange rounds)
  output files ....... main.cpp:634-713, Replica.cpp:1745-1777

The reference's worker threads, CUDA streams and GPU count are replaced by one
handle that advances every replica of the system in one persistent sweep per
block; -t/-s/-g/-bx are accepted and ignored. Random numbers come from a
counter-based stream keyed by --seed (the reference seeds from the clock).
"""
from __future__ import annotations

import dataclasses
import math
import os
import re
import sys
import time
from typing import List, Optional, Tuple

import numpy as np

from .model import (BOUND_ENERGY, AminoAcidTable, Molecule, ModelError, System, f32,
                    geometric_ladder, normalise_axis, reference_step_ladder)

# definitions.h:71-87 defaults
MC_STEPS = 5000
REMC_STEPS = 10
REPLICA_COUNT = 20
LOWTEMP = 250.0
HIGHTEMP = 500.0
BOUNDING_VALUE = 150.0


@dataclasses.dataclass
class Args:
    """argdata (definitions.h:203-225)."""
    threads: int = 1
    streams: int = 1
    gpus: int = 1
    mcsteps: int = MC_STEPS
    resteps: int = REMC_STEPS
    replicas: int = REPLICA_COUNT
    bound: float = BOUNDING_VALUE
    sample_frequency: int = MC_STEPS
    sample_after: int = MC_STEPS
    prefix: str = ""
    file: str = ""
    logfile: str = ""
    input_file: bool = False
    noncrowders: int = 0
    tmin: float = LOWTEMP
    tmax: float = HIGHTEMP
    pid: int = 0
    check: bool = False
    view: bool = False
    nosim: bool = False
    resume: str = ""
    seed: Optional[int] = None
    sensitivity: bool = False
    # width (kcal/mol) of the kernel that estimates the bound threshold's term
    sensitivity_bandwidth: float = 0.25
    autotune: bool = False     # pick threads, layout and cluster size by probe sweeps
    checkpoint_every: int = 0  # MC steps between checkpoints (0: off)
    checkpoint_dir: str = "checkpoints"
    output_dir: str = "output"
    data_dir: str = "data"
    files: List[Tuple[str, bool]] = dataclasses.field(default_factory=list)


class ArgError(ValueError):
    pass


def parse_cli(argv: List[str], a: Optional[Args] = None) -> Args:
    """getArgs (main.cpp:193-381); unknown flags are skipped as there."""
    a = a or Args()
    i = 0

    def val():
        if i + 1 >= len(argv):
            raise ArgError("missing value after %s" % argv[i])
        return argv[i + 1]

    while i < len(argv):
        t = argv[i]
        if t in ("-v", "--view"):
            a.view = True
            i += 1
        elif t in ("-q", "--nosim"):
            a.nosim = True
            i += 1
        elif t in ("-c",):
            a.check = True
            i += 1
        elif t in ("-bx", "--blockdim", "-t", "--threads", "-s", "--streams", "-g", "--gpus"):
            v = int(val())
            if t in ("-t", "--threads"):
                a.threads = v
            elif t in ("-s", "--streams"):
                a.streams = v
            elif t in ("-g", "--gpus"):
                a.gpus = v
            i += 2
        elif t in ("-f", "--file"):
            a.file = val()
            a.input_file = True
            i += 2
        elif t in ("-m", "--mcsteps"):
            a.mcsteps = int(val())
            i += 2
        elif t in ("-e", "--resteps"):
            a.resteps = int(val())
            i += 2
        elif t in ("-r", "--replicas"):
            a.replicas = int(val())
            i += 2
        elif t in ("-o", "--output"):
            a.logfile = val()
            i += 2
        elif t in ("-b", "--boundry"):
            a.bound = float(f32(float(val())))
            i += 2
        elif t in ("-t0", "--tmin"):
            a.tmin = float(f32(float(val())))
            i += 2
        elif t in ("-t1", "--tmax"):
            a.tmax = float(f32(float(val())))
            i += 2
        elif t in ("-z", "--resume"):
            a.resume = val()
            i += 2
        elif t == "--seed":
            a.seed = int(val())
            i += 2
        elif t == "--checkpoint-every":
            a.checkpoint_every = int(val())
            i += 2
        elif t == "--checkpoint-dir":
            a.checkpoint_dir = val()
            i += 2
        elif t == "--sensitivity":
            a.sensitivity = True
            i += 1
        elif t == "--sensitivity-bandwidth":
            a.sensitivity_bandwidth = float(val())
            i += 2
        elif t == "--autotune":
            a.autotune = True
            i += 1
        elif t == "--output-dir":
            a.output_dir = val()
            i += 2
        elif t == "--data-dir":
            a.data_dir = val()
            i += 2
        elif t in ("-h", "--help"):
            raise ArgError(USAGE)
        else:
            i += 1
    return a


USAGE = ("Usage: python -m remcdockingsimulator_b200 -f <filename> [-c] [-h] [-v] [-q] [-t x] "
         "[-s x] [-g x] [-m x] [-e x] [-r x] [-o x] [-b x] [-t0 x] [-t1 x] [-bx x] "
         "[-z checkpoint] [--seed x] [--sensitivity] [--sensitivity-bandwidth h] [--autotune] "
         "[--checkpoint-every steps] "
         "[--checkpoint-dir d] [--output-dir d] [--data-dir d]")

_PLACE = re.compile(r"^([tp])\(\s*([^,()]+),\s*([^,()]+),\s*([^,()]+)\)\s*"
                    r"r\(\s*([^,()]+),\s*([^,()]+),\s*([^,()]+),\s*([^,()]+)\)\s*(\S+)")


def _f(s: str) -> float:
    return float(f32(float(s)))


def load_config(a: Args, table: AminoAcidTable, log=print) -> List[Molecule]:
    """loadArgsFromFile (main.cpp:383-632): parameters, then the `files`
    section, then `crowders`, each line `t|p(x,y,z) r(ax,ay,az,angle) path`."""
    with open(a.file) as fh:
        lines = [ln.rstrip("\r\n")[:511] for ln in fh]
    section = "params"
    mols: List[Molecule] = []
    for lc, line in enumerate(lines, 1):
        toks = line.split()
        if not toks or line.startswith("#"):
            continue
        tok = toks[0]
        if tok == "files":
            section = "files"
            continue
        if tok == "crowders":
            section = "crowders"
            continue
        if section == "params":
            v = toks[1] if len(toks) > 1 else "0"
            if tok == "gpus":
                a.gpus = int(v)
            elif tok == "streams":
                a.streams = int(v)
            elif tok == "threads":
                a.threads = int(v)
            elif tok == "mcsteps":
                a.mcsteps = int(v)
            elif tok == "resteps":
                a.resteps = int(v)
            elif tok == "temperaturemax":
                a.tmax = _f(v)
            elif tok == "temperaturemin":
                a.tmin = _f(v)
            elif tok == "boundry":
                a.bound = _f(v)
            elif tok == "replicas":
                a.replicas = int(v)
            elif tok == "samplefrequency":
                a.sample_frequency = int(v)
            elif tok == "sampleafter":
                a.sample_after = int(v)
            elif tok == "prefix":
                a.prefix = v + "_repulsive"  # REPULSIVE_CROWDING build
            continue
        m = _PLACE.match(line)
        if not m:
            log("Failed to parse line %d: %s" % (lc, line))
            continue
        kind, px, py, pz, rx, ry, rz, ra, path = m.groups()
        mol = Molecule.from_pdb(path, table)
        v = np.array([_f(px), _f(py), _f(pz)], np.float32)
        if kind == "t":
            mol.translate(v)
        else:
            mol.set_position(v)
        ra_f = _f(ra)
        if ra_f >= 0.0:
            mol.rotate_q(normalise_axis(_f(rx), _f(ry), _f(rz)), ra_f)
        if section == "crowders":
            mol.crowder = True
        else:
            a.noncrowders += 1
        mol.name = path
        mols.append(mol)
        a.files.append((path, section == "crowders"))
    if a.bound <= 0:
        log("! Bounding value too small, setting equal to %g" % BOUNDING_VALUE)
    if a.tmax < a.tmin:
        log("! Maximum temperature < minimum temperature, swapping %g <-> %g" % (a.tmax, a.tmin))
        a.tmax, a.tmin = a.tmin, a.tmax
    if a.threads > a.replicas:
        a.threads = a.replicas
    return mols


def adjusted_sample_frequency(a: Args, log=print) -> int:
    """REMCSimulation's fit of the sampling interval to the exchange interval
    (main.cpp:1299-1316)."""
    per = a.mcsteps // a.resteps
    f = a.sample_frequency
    if f > 0 and per % f > 0:
        if per > f:
            while per % f != 0:
                f += 1
            log("-!- CHANGED: sample frequency <- %d. -!-" % f)
        if per < f:
            f = per
            log("-!- CHANGED: sample frequency <- %d. -!-" % f)
    return f


def _fmt_ratio(num: float, den: float) -> float:
    return num / den if den != 0 else float("nan")


class OutputFiles:
    """The four sampling files (main.cpp:634-713) plus the file index."""

    def __init__(self, a: Args, ladder: np.ndarray, header: bool = True):
        os.makedirs(a.output_dir, exist_ok=True)
        base = os.path.join(a.output_dir, "%s_%d" % (a.prefix, a.pid))
        self.fb = open(base + "_fractionBound", "a")
        self.bc = open(base + "_boundconformations", "a")
        self.ar = open(base + "_acceptance_ratios", "a")
        self.ex = open(base + "_exchange_freq", "a")
        self.base = base
        if not header:  # a resumed run appends to the files of the run it continues
            return
        self.fb.write("# Fraction Bound\n#Iteration InstantaniousAve CumulativeAve\n")
        self.bc.write("# iteration; complex free energy (replica free energy); temperature;\n"
                      "# molecule: rotation(w,x,y,z) position(x,y,z) 1 line per other molecule "
                      "in the bound state\n")
        self.ar.write("# Iteration AcceptanceRatio\n")
        self.ex.write("# Iteration continous_ratio, inst_ratio\n")
        self.fb.write("Iteration:  ")
        self.ar.write("Iteration:  ")
        for T in ladder:
            self.fb.write("%0.1fKi %0.1fKc " % (T, T))
            self.ar.write("%0.1fKi %0.1fKc " % (T, T))
        self.fb.write("\t\n")
        self.ar.write("\n")

    def flush(self):
        for f in (self.fb, self.bc, self.ar, self.ex):
            f.flush()

    def close(self):
        for f in (self.fb, self.bc, self.ar, self.ex):
            f.close()


# ------------------------------------------------------------------ checkpoints
CHECKPOINT_FREQUENCY = 10000  # definitions.h:116, MC steps between checkpoints

_CK_PARAMS = ("# threads, streams, gpus, MCsteps, RESteps, sampleFrequency, sampleStartsAfter,"
              "nonCrowders, temperatureMin, temperatureMax, currentStep")
_CK_STATS = ("stats: accept, acceptA, reject, totalAcceptReject, totalAccept, boundSamples, "
             "samplesSinceLastExchange, totalBoundSamples, totalSamples")
# driver accumulators saved with the engine state
_CK_ARRAYS = ("tot_bound", "tot_samples", "tot_acc", "tot_all", "pend_bound", "pend_samples",
              "pend_acc", "pend_accA", "pend_rej", "sens")


def checkpoint_path(a: Args) -> str:
    return os.path.join(a.checkpoint_dir, "%s_%d" % (a.prefix, a.pid))


def save_simulation(a: Args, path: str, blocks: int, seed: int, state, energies, ecc, tmap,
                    acc: dict, total_ex: int, total_tests: int) -> None:
    """saveSimulation (main.cpp:89-117): the reference's text layout (config
    file, prefix_pid, pid, run parameters with the current step, molecule and
    replica counts, then per replica slot one line per molecule with its
    position and rotation quaternion at %.7f and one statistics line), plus a
    line naming an .npz file with the exact engine state (coordinates, running
    energies, temperature map), the Philox seed and the driver's accumulators,
    from which a resumed run continues bit for bit."""
    pos, rel, cen, quat = state
    R = len(tmap)
    n_mol = cen.shape[0] // R
    per = a.mcsteps // a.resteps
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    npz = path + ".state.npz"
    tmp = npz + ".tmp.npz"
    np.savez(tmp, pos=pos, rel=rel, centre=cen, quat=quat, energies=energies, ecc=ecc,
             tmap=tmap, seed=np.uint64(seed), blocks=np.int64(blocks),
             total_ex=np.int64(total_ex), total_tests=np.int64(total_tests),
             **{k: acc[k] for k in _CK_ARRAYS})
    os.replace(tmp, npz)
    lines = ["#Saved simulation state file, prependage string, original pid", a.file,
             "%s_%d" % (a.prefix, a.pid), "%d" % a.pid, _CK_PARAMS,
             "%d %d %d %d %d %d %d %d %f %f %d" % (a.threads, a.streams, a.gpus, a.mcsteps,
                                                   a.resteps, a.sample_frequency, a.sample_after,
                                                   a.noncrowders, a.tmin, a.tmax, per * blocks),
             "#molecules", "%d" % n_mol, "#replicas", "%d" % R]
    for r in range(R):
        t = int(tmap[r])
        lines.append("#replica %d, molecules: x,y,z translation. w,x,y,z rotation quaternion" % r)
        for m in range(n_mol):
            c, q = cen[r * n_mol + m], quat[r * n_mol + m]
            lines.append("%.7f %.7f %.7f %.7f %.7f %.7f %.7f" % (c[0], c[1], c[2], q[0], q[1],
                                                                 q[2], q[3]))
        lines.append("#replica %d, %s" % (r, _CK_STATS))
        lines.append("%d %d %d %d %d %d %d %d %d" % (
            acc["pend_acc"][r], acc["pend_accA"][r], acc["pend_rej"][r], acc["tot_all"][t],
            acc["tot_acc"][t], acc["pend_bound"][r], acc["pend_samples"][r], acc["tot_bound"][t],
            acc["tot_samples"][t]))
    lines.append("#exact state %s" % os.path.basename(npz))
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    os.replace(tmp, path)


def read_checkpoint_header(path: str) -> dict:
    """The fields of a saved simulation that select the run to resume: the
    config file, prefix_pid, pid and the run parameters line."""
    with open(path) as fh:
        lines = [ln.rstrip("\n") for ln in fh]
    if len(lines) < 6 or not lines[0].startswith("#Saved simulation state"):
        raise ArgError("%s is not a saved simulation" % path)
    vals = lines[5].split()
    exact = [ln.split(None, 2)[2] for ln in lines if ln.startswith("#exact state ")]
    return {"file": lines[1], "prefix_pid": lines[2], "pid": int(lines[3]),
            "mcsteps": int(vals[3]), "resteps": int(vals[4]), "current_step": int(vals[10]),
            "replicas": int(lines[9]), "n_mol": int(lines[7]),
            "exact": os.path.join(os.path.dirname(os.path.abspath(path)), exact[0])
            if exact else None}


def load_simulation(path: str) -> dict:
    hdr = read_checkpoint_header(path)
    if hdr["exact"] is None or not os.path.exists(hdr["exact"]):
        raise ArgError("%s: exact state file missing" % path)
    with np.load(hdr["exact"]) as z:
        hdr.update({k: z[k] for k in z.files})
    return hdr


def write_file_index(a: Args) -> None:
    os.makedirs(a.output_dir, exist_ok=True)
    with open(os.path.join(a.output_dir, "%s_%d_fileindex" % (a.prefix, a.pid)), "w") as fh:
        fh.write("index molecule_file_path crowder(Y/N)\n")
        for i, (path, crowd) in enumerate(a.files):
            fh.write("%2d %s %s\n" % (i, path, "Y" if crowd else "N"))


def simulate(a: Args, system: System, params=None, log=print, on_checkpoint=None) -> dict:
    """REMCSimulation on the GPU engine. Returns summary statistics. With
    a.resume set, continues the run saved in that checkpoint; with
    a.checkpoint_every > 0, saves a checkpoint after every exchange round that
    completes that many MC steps (on_checkpoint(path, blocks) is called after
    each save)."""
    from .engine import Engine, make_params

    R = a.replicas
    ladder = geometric_ladder(a.tmin, a.tmax, R)
    tsteps, rsteps = reference_step_ladder(R)
    eng = Engine([system], R, params if params is not None else make_params())
    try:
        eng.set_replica_params([ladder], tsteps, rsteps)
        if a.autotune:
            # probe sweeps on a copy of the state; the state is restored after each
            t, m, c = eng.autotune(probe_steps=min(256, max(1, a.mcsteps // a.resteps)))[:2] + \
                (eng.schedule()[2],)
            log("Autotuned sweep: %d threads per replica, molecule data in %s memory, "
                "%d CTA(s) per replica" % (t, "shared" if m else "global", c))
        ck = load_simulation(a.resume) if a.resume else None
        if ck is None:
            e0 = eng.energy_full()
        else:
            if int(ck["replicas"]) != R or ck["pos"].shape[0] != R * system.n_beads:
                raise ArgError("checkpoint does not match this configuration")
            eng.upload_state(ck["pos"], ck["rel"], ck["centre"], ck["quat"])
            eng.set_temperature_map(ck["tmap"])
            eng.set_energies(ck["energies"], ck["ecc"])
            e0 = np.array(ck["energies"], np.float64)
        per = a.mcsteps // a.resteps
        if per <= 0:
            raise ArgError("mcsteps must be at least resteps")
        f = adjusted_sample_frequency(a, log)
        n_mol = system.n_mol
        max_rec = max(1, R * max(1, per // max(f, 1)))
        eng.set_sampling(f, a.sample_after, float(BOUND_ENERGY), max_rec, max_rec * n_mol)
        files = OutputFiles(a, ladder, header=ck is None)
        seed = a.seed if a.seed is not None else int(time.time())
        if ck is not None:
            seed = int(ck["seed"])
        # host mirror of the reference's per-replica statistics: slot counters
        # since the last report, cumulative totals that follow the temperature
        tot_bound = np.zeros(R, np.int64)
        tot_samples = np.zeros(R, np.int64)
        tot_acc = np.zeros(R, np.int64)
        tot_all = np.zeros(R, np.int64)
        pend_bound = np.zeros(R, np.int64)
        pend_samples = np.zeros(R, np.int64)
        pend_acc = np.zeros(R, np.int64)     # accept (dE < 0)
        pend_accA = np.zeros(R, np.int64)    # accept (Boltzmann)
        pend_rej = np.zeros(R, np.int64)
        last = [np.zeros(R, np.int64) for _ in range(5)]
        total_ex = total_tests = 0
        sens = SensitivitySums(R, a.sensitivity_bandwidth)  # per temperature
        has_crowders = system.n_chains < system.n_mol
        first_block = 1
        if ck is not None:
            for name, arr in (("tot_bound", tot_bound), ("tot_samples", tot_samples),
                              ("tot_acc", tot_acc), ("tot_all", tot_all),
                              ("pend_bound", pend_bound), ("pend_samples", pend_samples),
                              ("pend_acc", pend_acc), ("pend_accA", pend_accA),
                              ("pend_rej", pend_rej), ("sens", sens.sums)):
                arr[...] = ck[name]
            total_ex, total_tests = int(ck["total_ex"]), int(ck["total_tests"])
            first_block = int(ck["blocks"]) + 1
            log("Resuming after exchange round %d (step %d)" % (first_block - 1,
                                                                per * (first_block - 1)))
        ck_every = a.checkpoint_every
        until_ck = ck_every
        t0 = time.perf_counter()
        step0 = per * (first_block - 1)
        for steps in range(first_block, a.resteps + 1):
            if a.sensitivity:
                # one launch per sampling chunk (the same trajectory and the
                # same samples as one launch per block): B and X = dE/dlambda
                # at the end of every chunk past sampleafter, as
                # Replica::sample sees it (main.cpp:975-989)
                for c in range(per // f):
                    eng.sweep(f, seed, step0 + c * f)
                    if step0 + c * f >= a.sample_after:
                        en = eng.energies()
                        enc = en + eng.noncrowder_energies() if has_crowders else en
                        sens.add(eng.temperature_map(), enc, eng.dE_dlambda(),
                                 2.0 if has_crowders else 1.0)
            else:
                eng.sweep(per, seed, step0)
            step0 += per
            n_s, n_b = eng.sample_counters()
            acc, accA, rej = eng.counters()
            cur = [np.asarray(x, np.int64) for x in (n_b, n_s, acc, accA, rej)]
            d = [c - l for c, l in zip(cur, last)]
            last = cur
            pend_bound += d[0]
            pend_samples += d[1]
            pend_acc += d[2]
            pend_accA += d[3]
            pend_rej += d[4]
            recs, poses, dropped = eng.read_samples()
            for r in sorted(recs, key=lambda r: (r["label"], r["inst"])):
                files.bc.write("%d; %0.5f (%0.5f); %0.1f\n" % (r["label"], r["e_noncrowder"],
                                                               r["e_total"], r["temperature"]))
                for k in range(r["n_mol"]):
                    p = poses[r["pose_offset"] + k]
                    files.bc.write("%d %2d: %f %f %f %f %f %f %f\n" % (
                        0 if k < a.noncrowders else 1, k, p[0], p[1], p[2], p[3], p[4], p[5],
                        p[6]))
            if dropped:
                log("-!- %d bound conformations did not fit the record buffer" % dropped)
            if steps == a.resteps:
                break
            tos = eng.temperature_map()
            slot_of = np.argsort(tos)
            if per * (steps - 1) >= a.sample_after:
                files.fb.write("%9d: " % (per * steps))
                files.ar.write("%9d: " % (per * steps))
                for t in range(R):
                    sl = slot_of[t]
                    frac = pend_bound[sl] / max(1.0, float(pend_samples[sl]))
                    tot_bound[t] += pend_bound[sl]
                    tot_samples[t] += pend_samples[sl]
                    files.fb.write("| %6.4f %6.4f " % (frac, _fmt_ratio(tot_bound[t],
                                                                       tot_samples[t])))
                    a_ok = pend_acc[sl] + pend_accA[sl]
                    a_all = a_ok + pend_rej[sl]
                    tot_acc[t] += a_ok
                    tot_all[t] += a_all
                    files.ar.write("| %6.4f %6.4f " % (_fmt_ratio(a_ok, a_all),
                                                       _fmt_ratio(tot_acc[t], tot_all[t])))
                    pend_bound[sl] = pend_samples[sl] = 0
                    pend_acc[sl] = pend_accA[sl] = pend_rej[sl] = 0
                files.fb.write("\n")
                files.ar.write("\n")
                files.fb.flush()
                files.ar.flush()
            offset = (steps - 1) & 1
            eng.exchange(seed, steps - 1, offset)
            tos2 = eng.temperature_map()
            swapped = np.flatnonzero(tos2 != tos)
            tests = len(range(offset, R - 1, 2))
            exchanges = len(swapped) // 2
            # exchangeReplicas swaps the pending sample counts with the temperature
            for t in range(offset, R - 1, 2):
                a_sl, b_sl = slot_of[t], slot_of[t + 1]
                if tos2[a_sl] != tos[a_sl]:
                    pend_bound[[a_sl, b_sl]] = pend_bound[[b_sl, a_sl]]
                    pend_samples[[a_sl, b_sl]] = pend_samples[[b_sl, a_sl]]
            total_ex += exchanges
            total_tests += tests
            files.ex.write("%10d %6.4f %6.4f\n" % (steps, _fmt_ratio(total_ex, total_tests),
                                                   _fmt_ratio(exchanges, tests)))
            log("Replica Exchange step %d of %d complete" % (steps, a.resteps))
            if ck_every > 0:
                until_ck -= per
                if until_ck <= 0:
                    until_ck = ck_every
                    files.flush()
                    path = checkpoint_path(a)
                    acc_state = {"tot_bound": tot_bound, "tot_samples": tot_samples,
                                 "tot_acc": tot_acc, "tot_all": tot_all,
                                 "pend_bound": pend_bound, "pend_samples": pend_samples,
                                 "pend_acc": pend_acc, "pend_accA": pend_accA,
                                 "pend_rej": pend_rej, "sens": sens.sums}
                    save_simulation(a, path, steps, seed, eng.download_state(), eng.energies(),
                                    eng.noncrowder_energies(), eng.temperature_map(), acc_state,
                                    total_ex, total_tests)
                    if on_checkpoint is not None:
                        on_checkpoint(path, steps)
        eng.sync()
        elapsed = time.perf_counter() - t0
        # final lines (main.cpp:1509-1538)
        tos = eng.temperature_map()
        slot_of = np.argsort(tos)
        files.fb.write("%9d: " % a.mcsteps)
        files.ar.write("%9d: " % a.mcsteps)
        for t in range(R):
            sl = slot_of[t]
            tot_bound[t] += pend_bound[sl]
            tot_samples[t] += pend_samples[sl]
            files.fb.write("| %6.4f %6.4f  " % (_fmt_ratio(pend_bound[sl], pend_samples[sl]),
                                                _fmt_ratio(tot_bound[t], tot_samples[t])))
            all_ = pend_acc[sl] + pend_accA[sl] + pend_rej[sl]
            files.ar.write("| %6.4f %6.4f " % (_fmt_ratio(pend_accA[sl], all_),
                                               _fmt_ratio(tot_acc[t], tot_all[t])))
        files.fb.write("\n")
        files.ar.write("\n")
        files.close()
        sensitivity = None
        if a.sensitivity:
            sensitivity = sensitivity_estimates(ladder, sens.sums)
            with open(files.base + "_sensitivity", "w") as fh:
                fh.write("# temperature samples <B> <X> -beta(<BX>-<B><X>) <dB/dlambda> "
                         "d<B>/dlambda  (B: bound, E_nc < %.4f kcal/mol; X = dE/dlambda, "
                         "kcal/mol; <dB/dlambda>: threshold term, Gaussian kernel of %.3g "
                         "kcal/mol)\n" % (float(BOUND_ENERGY), a.sensitivity_bandwidth))
                for T, n, b, x, cov, surf, d in sensitivity:
                    fh.write("%0.1f %d %.6f %.6f %.6e %.6e %.6e\n" % (T, n, b, x, cov, surf, d))
        energies = eng.energies()
        log("Simulation: %10.5f ms  (%d exchanges)" % (elapsed * 1000.0, a.resteps))
        return {"elapsed_s": elapsed, "replica_steps": R * per * a.resteps, "e0": e0,
                "sensitivity": sensitivity,
                "energies": energies, "temperature_of_slot": tos, "files": files.base,
                "fraction_bound": _fmt_ratio(tot_bound.sum(), tot_samples.sum())}
    finally:
        eng.close()


class SensitivitySums:
    """Per-temperature sums for the fluctuation estimate of d<B>/dlambda.

    B = 1{E_nc < -1.1844 kcal/mol} is the bound indicator of Replica::sample
    (Replica.cpp:1717-1780, definitions.h:84): E_nc is the potential, plus the
    chain-chain pair energy when the system has crowders. X = dE/dlambda comes
    from the adjoint. The energy is linear in lambda (eps = lambda (M - e0)
    enters each residue pair linearly and crowder terms do not depend on it),
    and the chain-chain energy is the residue-pair part of E, so
    dE_nc/dlambda = c X with c = 2 when crowders are present, else 1. In the
    canonical ensemble at each temperature

        d<B>/dlambda = <dB/dlambda> - beta (<B X> - <B><X>),

    and since B depends on lambda through E_nc, dB/dlambda = -delta(E_nc - thr)
    c X: a threshold term, estimated with a Gaussian kernel of width h,
    -(1/n) sum_i K_h(E_nc,i - thr) c X_i. Columns per temperature: n, sum B,
    sum X, sum B X, sum K_h(E_nc - thr) c X."""

    def __init__(self, n_temps: int, bandwidth: float = 0.25,
                 threshold: float = float(BOUND_ENERGY)):
        if not bandwidth > 0.0:
            raise ArgError("sensitivity bandwidth must be positive")
        self.sums = np.zeros((n_temps, 5))
        self.h = float(bandwidth)
        self.thr = float(threshold)

    def add(self, temp_of_slot, e_nc, X, c: float = 1.0) -> None:
        """One sample per slot: the temperature index it holds, its E_nc and
        its dE/dlambda."""
        t = np.asarray(temp_of_slot, np.int64)
        e = np.asarray(e_nc, np.float64)
        x = np.asarray(X, np.float64)
        B = (e < self.thr).astype(np.float64)
        u = (e - self.thr) / self.h
        K = np.exp(-0.5 * u * u) / (self.h * np.sqrt(2.0 * np.pi))
        cols = np.stack([np.ones_like(x), B, x, B * x, K * c * x], axis=1)
        np.add.at(self.sums, t, cols)


def sensitivity_estimates(ladder: np.ndarray, sums: np.ndarray):
    """d<B>/dlambda per temperature from SensitivitySums columns (n, sum B,
    sum X, sum B X, sum K c X), beta = 4184 / (R T) per kcal/mol. Returns
    (T, n, <B>, <X>, -beta (<BX> - <B><X>), <dB/dlambda>, d<B>/dlambda) rows;
    sums with four columns (no threshold term) give a zero threshold term."""
    out = []
    nan = float("nan")
    for t, T in enumerate(ladder):
        n, sb, sx, sbx = sums[t][:4]
        skx = sums[t][4] if len(sums[t]) > 4 else 0.0
        if n == 0:
            out.append((float(T), 0, nan, nan, nan, nan, nan))
            continue
        beta = 4184.0 / (float(np.float32(8.314472)) * float(T))
        mb, mx, mbx = sb / n, sx / n, sbx / n
        cov = -beta * (mbx - mb * mx)
        surf = -skx / n
        out.append((float(T), int(n), mb, mx, cov, surf, cov + surf))
    return out


def check_mode(data_dir: str, table: AminoAcidTable, log=print) -> List[Tuple[float, float]]:
    """-c (main.cpp:1652-1707): the 10 two-chain conformations
    data/conf{1..10}/1{a,b}.pdb in a 118.4 A box, energy from the batched
    engine and from the reference-ABI kernel (two independent GPU paths)."""
    import ctypes as C
    from .engine import Engine, make_params
    from .reference_abi import abi, pack_reference_layout
    import torch
    out = []
    for i in range(1, 11):
        mols = [Molecule.from_pdb(os.path.join(data_dir, "conf%d" % i, n), table)
                for n in ("1a.pdb", "1b.pdb")]
        s = System(mols, 118.4, table)
        with Engine([s], 1, make_params()) as eng:
            e1 = float(eng.energy_full()[0])
        L = abi()
        pos, meta = pack_reference_layout(s, 64)
        dp, dm = torch.from_numpy(pos).cuda(), torch.from_numpy(meta).cuda()
        dt = torch.from_numpy(np.ascontiguousarray(table.pairs, np.float32).reshape(-1)).cuda()
        L.CUDA_setBoxDimension(118.4)
        r = C.c_double()
        L.CUDA_EonDevice(C.c_void_p(dp.data_ptr()), C.c_void_p(dm.data_ptr()), None, None, None,
                         C.c_void_p(dt.data_ptr()), C.byref(r), 64, pos.shape[0], 0)
        log("ENGINE,REFABI,err: %24.20f %24.20f %24.20f" % (e1, r.value, abs(e1 - r.value)))
        out.append((e1, r.value))
    return out


def main(argv: Optional[List[str]] = None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    try:
        a = parse_cli(argv)
    except ArgError as e:
        print(e)
        return 0
    a.pid = os.getpid()
    if a.resume:
        # getArgs -z (main.cpp:351-368): the config file and pid come from the
        # checkpoint, so the output files continue under the original name
        hdr = read_checkpoint_header(a.resume)
        a.file, a.pid, a.input_file = hdr["file"], hdr["pid"], True
    table = AminoAcidTable.load(os.path.join(a.data_dir, "AminoAcids"))
    table.load_pairs(os.path.join(a.data_dir, "pair_potentials_MJ1996"))
    if a.check:
        check_mode(a.data_dir, table)
        return 0
    if a.view:
        print("!!! This build does not support OpenGL and the -v option")
    if not a.input_file:
        print("No arguments.")
        print(USAGE)
        return 0
    mols = load_config(a, table)
    parse_cli(argv, a)  # second pass: flags override the file (main.cpp:1718)
    write_file_index(a)
    if not mols:
        print("-!- No molecules loaded. -!-")
        return 1
    system = System(mols, a.bound, table)
    print("Loaded: %d residues in %d molecules" % (system.n_beads, system.n_mol))
    if a.nosim:
        return 0
    summary = simulate(a, system)
    print("Output files will be prefixed by %s" % summary["files"])
    return 0


if __name__ == "__main__":
    sys.exit(main())
