"""Generate tests/golden/structures.json from the reference's known-answer data.

Run here, where the reference tree is mounted (it is read, never copied):
    python tests/golden/make_golden.py

Sources (paths inside iantunbridge/RemcDockingSimulator):
  post processor/data/structures.tgz           10 two-chain CA structures (1x..10x.pdb,
                                                chain split by segID column 73)
  simulation engine/data/AminoAcids            residue radii and charges
  simulation engine/data/pair_potentials_MJ1996 raw contact table
  simulation engine/data/structures/energy.txt  older totals of the reference code (col 2)
  simulation engine/data/structures/ref_ene_nocut_noim_c35a2.dat
                                                an independent implementation's totals
  simulation engine/data/pairinteractions/pairs_N.dat
                                                per-pair (elec, vdw) values of that
                                                implementation; their sums are stored

Each structure's energy is also evaluated by the reference's own
Replica::E() (oracle/_ref, built from the reference sources) in the -c check
mode's 118.4 A box (main.cpp:1652-1707); those values pin the FP64 oracle
tightly. The JSON stores coordinates, types and the tables, so tests do not
need the reference tree.
"""
from __future__ import annotations

import io
import json
import os
import sys
import tarfile
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.build import reference_root  # noqa: E402

REF = reference_root()
SE = os.path.join(REF, "simulation engine")
PP = os.path.join(REF, "post processor")
BOX = 118.4


def main() -> int:
    from oracle import bindings as ob
    from remcdockingsimulator_b200.model import AminoAcidTable, Molecule, System

    table = AminoAcidTable.load(os.path.join(SE, "data", "AminoAcids"))
    table.load_pairs(os.path.join(SE, "data", "pair_potentials_MJ1996"))

    # older totals (col 2) and the independent implementation (ref_ene)
    energy_txt = {}
    with open(os.path.join(SE, "data", "structures", "energy.txt")) as fh:
        for ln in fh:
            if ln.startswith("#") or not ln.strip():
                continue
            t = ln.split()
            energy_txt[int(t[0])] = [float(x) for x in t[1:7]]
    pair_sums = {}
    for k in range(1, 11):
        tot = elec = vdw = 0.0
        n = 0
        with open(os.path.join(SE, "data", "pairinteractions", "pairs_%d.dat" % k)) as fh:
            for ln in fh:
                t = ln.split()
                if len(t) < 5:
                    continue
                tot += float(t[2])
                elec += float(t[3])
                vdw += float(t[4])
                n += 1
        pair_sums[k] = {"total": tot, "elec": elec, "vdw": vdw, "pairs": n}

    out = {"box": BOX, "table": {"names": table.names, "snames": table.snames,
                                 "symbols": table.symbols, "vdw": table.vdw.tolist(),
                                 "charge": table.charge.tolist(),
                                 "pairs": table.pairs.tolist()},
           "structures": []}
    tmp = tempfile.mkdtemp()
    with tarfile.open(os.path.join(PP, "data", "structures.tgz")) as tf:
        for k in range(1, 11):
            member = [m for m in tf.getmembers() if m.name.endswith("/%dx.pdb" % k) or
                      m.name == "%dx.pdb" % k or m.name.endswith("%dx.pdb" % k)][0]
            text = tf.extractfile(member).read().decode("latin-1")
            chains = {}
            for ln in text.splitlines():
                if ln.startswith("ATOM"):
                    seg = ln[72:76].strip() or "A"
                    chains.setdefault(seg, []).append(ln)
            mols = []
            for seg in sorted(chains):
                path = os.path.join(tmp, "%d_%s.pdb" % (k, seg))
                with open(path, "w") as fh:
                    fh.write("\n".join(chains[seg]) + "\nEND\n")
                mols.append(Molecule.from_pdb(path, table))
            sysm = System(mols, BOX, table)
            ref = ob.ReferenceReplica(sysm)
            e_ref = ref.E()
            e_pair = ref.E_pair(0, 1)
            ref.close()
            out["structures"].append({
                "index": k,
                "chains": [{"types": m.types.tolist(), "pos": m.pos.tolist()} for m in mols],
                "reference_E": e_ref,
                "reference_E_pair": e_pair,
                "energy_txt_total": energy_txt[k][0],
                "independent_total": energy_txt[k][3],
                "pair_file_sums": pair_sums[k],
            })
            print(k, [m.n for m in mols], e_ref, energy_txt[k][0], energy_txt[k][3])
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "structures.json")
    with open(dst, "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", dst)
    return 0


if __name__ == "__main__":
    sys.exit(main())
