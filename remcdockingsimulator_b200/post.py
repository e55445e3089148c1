"""Post-processing of REMC output on the GPU: bound-pose extraction and DRMS.

  python -m remcdockingsimulator_b200.post pdbgen <prefix_pid_fileindex> <box> [0|1 reverse]
         [0|1 crowders] [--temperature T] [--min-iteration N] [--data-dir d] [--out-dir d]
  python -m remcdockingsimulator_b200.post traj <trajectory.pdb> <reference list> <molecules>
         <length 1> ... [--box L] [--data-dir d]

pdbgen mirrors the reference's pose extractor (post processor/pdbgensrc/
pdbgen.cpp): it reads the run's file index and _boundconformations, keeps the
samples near `--temperature` (300 K) after `--min-iteration` steps (the
reference's 10,000,000), rebuilds every kept sample's bead coordinates from
its poses on the GPU (remc_post_rebuild) and writes one PDB per sample in
Replica::saveAsSinglePDB's layout (Replica.cpp:495-530) into
`pdbgen_results/`. It also writes `<prefix>drms.dat` with the energy and the
DRMS of every kept sample against the loaded conformation (the reference
computes the same DRMS, drms.cpp:7-57, with its output commented out).

traj mirrors the reference's trajectory post-processor (post processor/
postprocess/main.cpp:293-429): every frame of a multi-model CA trajectory is
split into molecules of the given lengths; its DRMS against the reference
structures (molecule order reversed too, keeping the smaller) and its energy
(the batched engine's full energy, frames as replicas) go to
`<trajectory>.drms.dat`, and the frames to `<trajectory>.delim.pdb`.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import sys
from typing import List, Optional, Sequence

import numpy as np

from ._capi import check, lib
from .model import AminoAcidTable, Molecule, ModelError, System

MIN_ITERATION = 10_000_000  # pdbgen.cpp:173
NATIVE_CUT = 12.0           # main.cpp:812 (12 Angstrom; the reference's unit constant makes it 1.2e-9)
RECOVERED_CUT = 15.0        # main.cpp:815


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def rebuild(molecules: Sequence[Molecule], shift: Sequence[int], box: float, quat: np.ndarray,
            centre: np.ndarray):
    """Bead coordinates [frames, beads, 3] (and the shifted centres
    [frames, molecules, 3]) of molecules placed at the given poses, from their
    loaded relative positions (remc_post_rebuild)."""
    rel0 = np.ascontiguousarray(np.concatenate([m.rel for m in molecules]), np.float32)
    ms = np.zeros(len(molecules) + 1, np.int32)
    for k, m in enumerate(molecules):
        ms[k + 1] = ms[k] + m.n
    sh = np.ascontiguousarray(shift, np.int32)
    c0 = np.ascontiguousarray(molecules[0].centre, np.float32)
    q = np.ascontiguousarray(quat, np.float64)
    c = np.ascontiguousarray(centre, np.float32)
    nf = q.shape[0]
    pos = np.zeros((nf, int(ms[-1]), 3), np.float32)
    cout = np.zeros((nf, len(molecules), 3), np.float32)
    check(lib().remc_post_rebuild(_f(rel0), _i(ms), len(molecules), _i(sh), _f(c0),
                                  C.c_float(box), _d(q), _f(c), nf, _f(pos), _f(cout)))
    return pos, cout


def drms(frames: np.ndarray, ref: np.ndarray, mol_start: np.ndarray, reverse: bool = False,
         native_cut: float = NATIVE_CUT, recovered_cut: float = RECOVERED_CUT):
    """DRMS of every frame against ref, and the contact counts (native,
    recovered, binding) per frame (remc_post_drms)."""
    x = np.ascontiguousarray(frames, np.float32)
    r = np.ascontiguousarray(ref, np.float32)
    ms = np.ascontiguousarray(mol_start, np.int32)
    nf = x.shape[0]
    out = np.zeros(nf)
    counts = [np.zeros(nf, np.int64) for _ in range(3)]
    P = [c.ctypes.data_as(C.POINTER(C.c_longlong)) for c in counts]
    check(lib().remc_post_drms(_f(x), nf, _f(r), _i(ms), len(ms) - 1, 1 if reverse else 0,
                               C.c_float(native_cut), C.c_float(recovered_cut), _d(out), *P))
    return out, counts[0], counts[1], counts[2]


# ------------------------------------------------------------------ pdbgen
_HEADER = re.compile(r"^\s*(-?\d+);\s*(\S+)\s*\(\s*(\S+)\s*\);\s*(\S+)")
_POSE = re.compile(r"^\s*(\d+)\s+(\d+):\s*(.*)$")


def read_index(path: str):
    """(path, crowder) per line of a run's _fileindex (main.cpp:714-721)."""
    out = []
    with open(path) as fh:
        for ln in fh:
            t = ln.split()
            if len(t) >= 3 and re.match(r"^-?\d+$", t[0]) and t[2] in ("Y", "N"):
                out.append((t[1], t[2] == "Y"))
    return out


def read_bound_conformations(path: str):
    """Samples of a _boundconformations file: (iteration, energy, replica
    energy, temperature, poses) with poses [(crowder, index, w, x, y, z, px,
    py, pz)] (Replica.cpp:1745-1777 writes them)."""
    samples = []
    with open(path) as fh:
        for ln in fh:
            m = _HEADER.match(ln)
            if m:
                samples.append((int(m.group(1)), float(m.group(2)), float(m.group(3)),
                                float(m.group(4)), []))
                continue
            p = _POSE.match(ln)
            if p and samples:
                vals = [float(v) for v in p.group(3).split()[:7]]
                if len(vals) == 7:
                    samples[-1][4].append((int(p.group(1)), int(p.group(2)), *vals))
    return samples


def save_as_single_pdb(path: str, molecules: Sequence[Molecule], pos: np.ndarray,
                       table: AminoAcidTable, potential: float, temperature: float,
                       quat: np.ndarray, centre: np.ndarray) -> None:
    """Replica::saveAsSinglePDB (Replica.cpp:495-530): remarks with the
    potential, temperature and each molecule's pose, CA atoms chain by chain."""
    lines = ["REMARK %s " % path, "REMARK potential: %0.10f " % np.float32(potential),
             "REMARK temperature: %5.1f " % temperature]
    for i in range(len(molecules)):
        q, c = quat[i], centre[i]
        lines.append("REMARK Molecule: %d" % i)
        lines.append("REMARK Rotation relative to input Q(w,x,y,z): %f %f %f %f" % tuple(q))
        lines.append("REMARK Centriod position P(x,y,z): %f %f %f" % tuple(c))
    chain = ord("A")
    item = 0
    b = 0
    for m in molecules:
        seq = m.res_seq if m.res_seq is not None else np.arange(1, m.n + 1)
        last = 0
        for k in range(m.n):
            item += 1
            x, y, z = pos[b]
            lines.append("ATOM  %5d %4s%c%3s %c%4d%c  %8.3f%8.3f%8.3f%6.2f%6.2f" % (
                item, "CA", " ", table.snames[int(m.types[k])], chr(chain), int(seq[k]), " ", x, y,
                z, 1.0, 1.0))
            last = int(seq[k])
            b += 1
        lines.append("TER   %5d      %3s %c%4d " % (item, table.snames[int(m.types[-1])], chr(chain),
                                                    last))
        chain += 1
    lines.append("END ")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def pdbgen(index_path: str, box: float, reverse: bool = False, crowders: bool = False,
           temperature: float = 300.0, min_iteration: int = MIN_ITERATION,
           data_dir: str = "data", out_dir: str = "pdbgen_results", log=print) -> dict:
    """pdbgen (pdbgen.cpp:19-235) with the rebuild and the DRMS on the GPU."""
    if "fileindex" not in index_path:
        raise ValueError("You must provide an index file as the input")
    table = AminoAcidTable.load(os.path.join(data_dir, "AminoAcids"))
    table.load_pairs(os.path.join(data_dir, "pair_potentials_MJ1996"))
    entries = read_index(index_path)
    mols: List[Molecule] = []
    is_crowd: List[bool] = []
    for path, crowd in entries:
        if not crowd or crowders:
            mols.append(Molecule.from_pdb(path, table))
            is_crowd.append(crowd)
    if not mols:
        raise ModelError("no molecules to rebuild")
    base = index_path[:index_path.rindex("fileindex")]
    samples = read_bound_conformations(base + "boundconformations")
    keep = [s for s in samples if abs(s[3] - temperature) < 1.0 and s[0] > min_iteration]
    n_mol = len(mols)
    quat = np.zeros((len(keep), n_mol, 4))
    cen = np.zeros((len(keep), n_mol, 3), np.float32)
    for f, s in enumerate(keep):
        poses = [p for p in s[4] if p[0] == 0 or crowders]
        if len(poses) < n_mol:
            raise ModelError("sample at iteration %d has %d poses for %d molecules" %
                             (s[0], len(poses), n_mol))
        for i in range(n_mol):
            quat[f, i] = poses[i][2:6]
            cen[f, i] = poses[i][6:9]
    shift = [0 if c else 1 for c in is_crowd]
    summary = {"samples": len(samples), "kept": len(keep), "files": [], "drms": None}
    if not keep:
        return summary
    pos, cout = rebuild(mols, shift, box, quat, cen)
    ms = np.zeros(n_mol + 1, np.int32)
    for k, m in enumerate(mols):
        ms[k + 1] = ms[k] + m.n
    ref = np.concatenate([m.pos for m in mols]).astype(np.float32)
    d = drms(pos, ref, ms, reverse=reverse)[0] if n_mol > 1 else np.zeros(len(keep))
    os.makedirs(out_dir, exist_ok=True)
    for f, s in enumerate(keep):
        # the rotation each molecule holds after setRotation: q * identity
        qn = quat[f] / np.linalg.norm(quat[f], axis=1, keepdims=True)
        name = os.path.join(out_dir, "sample_%d_%0.1fK_%5.2f.pdb" % (f + 1, s[3], s[1]))
        save_as_single_pdb(name, mols, pos[f], table, s[1], s[3], qn, cout[f])
        summary["files"].append(name)
        log("Saved frame %d: %s" % (f + 1, name))
    with open(base + "drms.dat", "w") as fh:
        for s, v in zip(keep, d):
            fh.write("%.7g %.7g\n" % (s[1], v))
    summary["drms"] = d
    summary["positions"] = pos
    return summary


# ------------------------------------------------------------------ trajectories
def _scan(s: str) -> float:
    m = re.match(r"\s*[-+]?(\d+\.?\d*|\.\d+)([eE][-+]?\d+)?", s)
    return float(np.float32(float(m.group(0)))) if m else 0.0


def read_trajectory(path: str, lengths: Sequence[int], table: AminoAcidTable):
    """Frames of a multi-model CA trajectory, split into molecules of the
    given lengths (extractMolecule, postprocess/main.cpp:92-249): ATOM lines
    named CA, coordinates from columns 31-54, other records skipped."""
    per = int(sum(lengths))
    types: List[int] = []
    xyz: List[List[float]] = []
    frames, frame_types = [], []
    with open(path) as fh:
        for ln in fh:
            if ln.split(" ", 1)[0] != "ATOM":
                continue
            name = ln[12:16].split()
            if not name or name[0] != "CA":
                continue
            res = ln[17:20].split()
            t = table.index(res[0] if res else "")
            if t < 0:
                raise ModelError("%s: unknown residue name %r" % (path, ln[17:20]))
            xyz.append([_scan(ln[30:38]), _scan(ln[38:46]), _scan(ln[46:54])])
            types.append(t)
            if len(xyz) == per:
                frames.append(np.array(xyz, np.float32))
                frame_types.append(np.array(types, np.int32))
                xyz, types = [], []
    return frames, frame_types


def process_trajectory(traj_path: str, reference_list: str, lengths: Sequence[int],
                       box: float = 150.0, data_dir: str = "data", params=None, log=print):
    """The trajectory post-processor: per frame DRMS (reverse order too) and
    energy, written to <traj>.drms.dat and <traj>.delim.pdb."""
    from .engine import Engine, make_params
    table = AminoAcidTable.load(os.path.join(data_dir, "AminoAcids"))
    table.load_pairs(os.path.join(data_dir, "pair_potentials_MJ1996"))
    with open(reference_list) as fh:
        ref_mols = [Molecule.from_pdb(ln.strip(), table) for ln in fh if ln.strip()]
    frames, ftypes = read_trajectory(traj_path, lengths, table)
    if not frames:
        raise ModelError("%s: no complete frame" % traj_path)
    ms = np.zeros(len(lengths) + 1, np.int32)
    ms[1:] = np.cumsum(lengths)
    ref = np.concatenate([m.pos for m in ref_mols]).astype(np.float32)
    if ref.shape[0] != ms[-1]:
        raise ModelError("reference structures have %d beads, frames %d" % (ref.shape[0], ms[-1]))
    X = np.stack(frames)
    d = drms(X, ref, ms, reverse=True)[0]
    # energies: frames as replicas of one system (Replica::EonDevice per frame)
    mols = [Molecule.from_beads(ftypes[0][ms[k]:ms[k + 1]], frames[0][ms[k]:ms[k + 1]])
            for k in range(len(lengths))]
    system = System(mols, box, table)
    nf = len(frames)
    with Engine([system], nf, params if params is not None else make_params()) as eng:
        pos = X.reshape(-1, 3)
        rel = np.zeros_like(pos)
        cen = np.zeros((nf * len(lengths), 3), np.float32)
        quat = np.tile(np.array([1.0, 0.0, 0.0, 0.0]), (nf * len(lengths), 1))
        eng.upload_state(pos, rel, cen, quat)
        energies = eng.energy_full()
    with open(traj_path + ".drms.dat", "w") as fh:
        for e, v in zip(energies, d):
            fh.write("%.6g\t%.6g\n" % (e, v))
    with open(traj_path + ".delim.pdb", "w") as fh:
        for f in range(nf):
            fh.write("TITLE     frame t=%7.3f\n" % float(f + 1))
            fh.write("MODEL%9d\n" % (f + 1))
            fh.write("REMARK potential,drms: %0.10f %0.10f \n" % (energies[f], d[f]))
            b = 0
            item = 0
            for k, L in enumerate(lengths):
                chain = chr(ord("A") + k)
                for r in range(L):
                    item += 1
                    x, y, z = frames[f][b]
                    fh.write("ATOM  %5d %4s%c%3s %c%4d%c  %8.3f%8.3f%8.3f%6.2f%6.2f\n" % (
                        item, "CA", " ", table.snames[int(ftypes[f][b])], chain, r + 1, " ", x, y,
                        z, 1.0, 1.0))
                    b += 1
                fh.write("TER   %5d      %3s %c%4d \n" % (item, table.snames[int(ftypes[f][b - 1])],
                                                         chain, L))
            fh.write("ENDMDL\n")
    log("Finished.")
    return {"frames": nf, "drms": d, "energies": energies}


def main(argv: Optional[List[str]] = None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    opts = {"--temperature": 300.0, "--min-iteration": MIN_ITERATION, "--data-dir": "data",
            "--out-dir": "pdbgen_results", "--box": 150.0}
    pos_args: List[str] = []
    i = 0
    while i < len(argv):
        if argv[i] in opts and i + 1 < len(argv):
            opts[argv[i]] = type(opts[argv[i]])(argv[i + 1])
            i += 2
        else:
            pos_args.append(argv[i])
            i += 1
    if len(pos_args) >= 3 and pos_args[0] == "pdbgen":
        reverse = len(pos_args) > 3 and pos_args[3].startswith("1")
        crowd = len(pos_args) > 4 and pos_args[4].startswith("1")
        s = pdbgen(pos_args[1], float(pos_args[2]), reverse, crowd, opts["--temperature"],
                   int(opts["--min-iteration"]), opts["--data-dir"], opts["--out-dir"])
        print("kept %d of %d samples" % (s["kept"], s["samples"]))
        return 0
    if len(pos_args) >= 5 and pos_args[0] == "traj":
        n = int(pos_args[3])
        lengths = [int(x) for x in pos_args[4:4 + n]]
        s = process_trajectory(pos_args[1], pos_args[2], lengths, opts["--box"], opts["--data-dir"])
        print("processed %d frames" % s["frames"])
        return 0
    print(__doc__)
    return 0


if __name__ == "__main__":
    sys.exit(main())
