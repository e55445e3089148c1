"""Seeded synthetic REMC workloads.

The reference ships no benchmark inputs (its performance_configs/ directory
and the application PDBs are absent), so these generators build systems with
the shapes, sizes and value distributions the benchmark configurations name:

  two_chain  76 + 24 residue chains, 100 A box, 20 replicas 290-450 K
  crowded    two_chain + 400 crowders (radius 12 A) in a 200 A box,
             r^-12 crowder walls, crowders translate only, 32 replicas 290-480 K
  batch64    64 systems of 2-8 chains x 20-300 residues and 0-1000 crowders,
             box sized for packing fraction 0.1-0.3, 16 replicas each
  assembly   60 x 150-residue chains + 2000 crowders (radius 10 A) in a
             400 A box, 32 replicas 290-500 K

Chains are compact self-avoiding random walks with 3.8 A bonds and no
non-bonded pair closer than 3.8 A; residue types are uniform over the 20
types (K/R +1, D/E -1); the contact matrix is U[-1.2, 0.2] kT, symmetrised;
sigma = 6 A for every residue, lambda = 0.16, Debye length 10 A. Every system
can be written out in the reference's own config / PDB / table formats
(`write_reference_inputs`) so the reference CPU engine runs the same input.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional

import numpy as np

from .engine import make_params
from .model import (CROWDER_TYPE, AminoAcidTable, Molecule, System, geometric_ladder,
                    write_pdb_ca)

BOND = 3.8
MIN_SEP = 3.8
RESIDUE_RADIUS = 3.0  # sigma / 2 for sigma = 6 A


@dataclasses.dataclass
class Workload:
    name: str
    systems: List[System]
    n_replicas: List[int]
    ladders: List[np.ndarray]
    translate_step: float
    rotate_step: float
    params: object
    mc_steps: int
    steps_per_exchange: int
    description: str = ""

    @property
    def n_inst(self) -> int:
        return int(sum(self.n_replicas))


def contact_table(rng: np.random.Generator, lambda_: float = 0.16, e0: float = -2.27,
                  lo: float = -1.2, hi: float = 0.2) -> AminoAcidTable:
    """Synthetic residue table with eps ~ U[lo, hi] symmetrised; stored as the
    raw table M = eps / lambda + e0 so that lambda (M - e0) = eps."""
    t = AminoAcidTable.synthetic(vdw=6.0)
    eps = rng.uniform(lo, hi, size=(20, 20))
    eps = np.triu(eps) + np.triu(eps, 1).T
    t.pairs = (eps / lambda_ + e0).astype(np.float32)
    return t


def compact_chain(rng: np.random.Generator, n: int, n_cand: int = 24) -> np.ndarray:
    """Compact self-avoiding walk: each bead 3.8 A from the previous one, no
    non-bonded pair below 3.8 A; among valid candidate directions the one
    nearest the running centroid is kept (random among the best three)."""
    for _attempt in range(200):
        pos = np.zeros((n, 3))
        ok = True
        for i in range(1, n):
            d = rng.normal(size=(n_cand, 3))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            cand = pos[i - 1] + BOND * d
            if i >= 2:
                diff = cand[:, None, :] - pos[None, : i - 1, :]
                dmin = np.sqrt((diff ** 2).sum(-1)).min(axis=1)
                valid = dmin >= MIN_SEP
            else:
                valid = np.ones(n_cand, bool)
            if not valid.any():
                ok = False
                break
            cen = pos[:i].mean(axis=0)
            dist = np.linalg.norm(cand - cen, axis=1)
            dist[~valid] = np.inf
            order = np.argsort(dist)
            nvalid = int(valid.sum())
            pick = order[rng.integers(0, min(3, nvalid))]
            pos[i] = cand[pick]
        if ok:
            return (pos - pos.mean(axis=0)).astype(np.float32)
    raise RuntimeError("could not grow a %d-residue chain" % n)


def _min_image(d: np.ndarray, L: float) -> np.ndarray:
    return d - L * np.round(d / L)


def _random_axis(rng):
    v = rng.normal(size=3)
    v /= np.linalg.norm(v)
    return float(v[0]), float(v[1]), float(v[2])


def build_system(rng: np.random.Generator, table: AminoAcidTable, chains, n_crowders: int,
                 crowder_radius: float, box: float, translate_only_crowders: bool = True,
                 max_tries: int = 20000) -> System:
    """Place chains (random centre and orientation, no bead pair closer than
    3.8 A under minimum image), then crowders uniformly with overlaps
    rejected (crowder-crowder >= 2R, crowder-residue >= R + 3 A).
    `chains` holds chain lengths (a new random chain each) or prebuilt
    (types, xyz) pairs."""
    mols: List[Molecule] = []
    placed = np.zeros((0, 3))
    for spec in chains:
        if isinstance(spec, (int, np.integer)):
            xyz = compact_chain(rng, int(spec))
            types = rng.integers(0, 20, size=int(spec))
        else:
            types, xyz = spec
        for _ in range(max_tries):
            m = Molecule.from_beads(types, xyz)
            m.set_position(rng.uniform(0.0, box, size=3).astype(np.float32))
            m.rotate_q(_random_axis(rng), float(rng.uniform(0.0, 2.0 * math.pi)))
            if placed.shape[0] == 0:
                break
            d = _min_image(m.pos[:, None, :].astype(np.float64) - placed[None, :, :], box)
            if np.sqrt((d ** 2).sum(-1)).min() >= MIN_SEP:
                break
        else:
            raise RuntimeError("could not place a chain without overlap")
        mols.append(m)
        placed = np.concatenate([placed, m.pos.astype(np.float64)])
    crowders = place_crowders(rng, n_crowders, crowder_radius, box, placed)
    for c in crowders:
        m = Molecule.from_beads([CROWDER_TYPE], np.zeros((1, 3), np.float32))
        m.crowder = True
        m.set_position(c.astype(np.float32))
        mols.append(m)
    return System(mols, float(np.float32(box)), table, crowder_radius=crowder_radius,
                  translate_only_crowders=translate_only_crowders)


def place_crowders(rng: np.random.Generator, n: int, radius: float, box: float,
                   residues: np.ndarray) -> np.ndarray:
    """Random sequential insertion of n spheres: each new centre is uniform
    over the space still free (crowder-crowder >= 2R, crowder-residue >= R + 3
    A, minimum image), drawn from a voxel map of the free space and checked
    exactly. Near the jamming density plain rejection sampling needs millions
    of draws per insertion; the voxel map keeps every draw likely to succeed."""
    if n == 0:
        return np.zeros((0, 3))
    h = 1.0 if box <= 150.0 else 2.0
    G = int(math.ceil(box / h))
    free = np.ones((G, G, G), bool)

    def stencil(excl: float) -> np.ndarray:
        # voxels lying wholly within distance excl of any point of the centre's voxel
        r = int(excl / h) + 1
        o = np.arange(-r, r + 1)
        ox, oy, oz = np.meshgrid(o, o, o, indexing="ij")
        off = np.stack([ox.ravel(), oy.ravel(), oz.ravel()], axis=1)
        keep = np.sqrt((off.astype(np.float64) ** 2).sum(1)) * h + math.sqrt(3.0) * h <= excl
        return off[keep]

    def block(p: np.ndarray, off: np.ndarray) -> None:
        v = np.floor(p / h).astype(np.int64) % G
        idx = (v[None, :] + off) % G
        free[idx[:, 0], idx[:, 1], idx[:, 2]] = False

    st_res = stencil(radius + RESIDUE_RADIUS)
    for p in residues:
        block(np.mod(p, box), st_res)
    st_cc = stencil(2.0 * radius)
    crowders = np.zeros((n, 3))
    count = 0
    free_idx = np.flatnonzero(free)
    K = 32
    while count < n:
        if free_idx.size == 0:
            raise RuntimeError("no free volume left after %d of %d crowders" % (count, n))
        # K draws, taken in order as sequential insertions
        ks = free_idx[rng.integers(0, free_idx.size, size=K)]
        v = np.stack(np.unravel_index(ks, free.shape), axis=1).astype(np.float64)
        cand = np.minimum((v + rng.uniform(0.0, 1.0, size=(K, 3))) * h, np.nextafter(box, 0.0))
        ok = np.ones(K, bool)
        if count:
            d = _min_image(cand[:, None, :] - crowders[None, :count, :], box)
            ok &= np.sqrt((d ** 2).sum(-1)).min(axis=1) >= 2.0 * radius
        if residues.shape[0]:
            d = _min_image(cand[:, None, :] - residues[None, :, :], box)
            ok &= np.sqrt((d ** 2).sum(-1)).min(axis=1) >= radius + RESIDUE_RADIUS
        first = count
        for i in np.flatnonzero(ok):
            if count >= n:
                break
            c = cand[i]
            if count > first:
                d = _min_image(crowders[first:count] - c[None, :], box)
                if np.sqrt((d ** 2).sum(-1)).min() < 2.0 * radius:
                    continue
            crowders[count] = c
            count += 1
            block(c, st_cc)
        if count - first < K // 4:
            # many draws hit voxels blocked since the list was made: refresh it
            free_idx = free_idx[free.ravel()[free_idx]]
    return crowders


def benchmark_params():
    # lambda = 0.16, Debye 10 A, r^-12 crowder walls with sigma = rho_i + rho_j, no cutoff
    return make_params(lambda_=0.16, e0=-2.27, debye_length=10.0, crowder_mode=1,
                       crowder_cutoff=0.0, crowder_eps=1.0)


def two_chain(seed: int = 0, mc_steps: int = 10_000) -> Workload:
    rng = np.random.default_rng(seed)
    table = contact_table(rng)
    s = build_system(rng, table, [76, 24], 0, 0.0, 100.0)
    R = 20
    return Workload("two_chain", [s], [R], [geometric_ladder(290.0, 450.0, R)], 0.5, 0.2,
                    benchmark_params(), mc_steps, 1000,
                    "76+24-residue chains, 100 A box, 20 replicas 290-450 K")


def crowded(seed: int = 0, mc_steps: int = 100_000) -> Workload:
    rng = np.random.default_rng(seed)
    table = contact_table(rng)
    s = build_system(rng, table, [76, 24], 400, 12.0, 200.0)
    R = 32
    return Workload("crowded", [s], [R], [geometric_ladder(290.0, 480.0, R)], 0.5, 0.2,
                    benchmark_params(), mc_steps, 1000,
                    "76+24 chains + 400 crowders R=12 A, 200 A box, 32 replicas 290-480 K")


def batch64(seed: int = 0, n_systems: int = 64, mc_steps: int = 10_000) -> Workload:
    rng = np.random.default_rng(seed)
    table = contact_table(rng)
    systems, ladders = [], []
    R = 16
    crowder_radius = 12.0
    for _ in range(n_systems):
        n_chains = int(rng.integers(2, 9))
        lengths = [int(rng.integers(20, 301)) for _ in range(n_chains)]
        n_crowd = int(rng.integers(0, 1001))
        phi = float(rng.uniform(0.1, 0.3))
        vol = (n_crowd * 4.0 / 3.0 * math.pi * crowder_radius ** 3 +
               sum(lengths) * 4.0 / 3.0 * math.pi * RESIDUE_RADIUS ** 3)
        box = max((vol / phi) ** (1.0 / 3.0), 80.0)
        systems.append(build_system(rng, table, lengths, n_crowd, crowder_radius, box))
        ladders.append(geometric_ladder(290.0, 450.0, R))
    return Workload("batch64", systems, [R] * n_systems, ladders, 0.5, 0.2, benchmark_params(),
                    mc_steps, 1000,
                    "%d systems: 2-8 chains x 20-300 residues, 0-1000 crowders R=12 A, "
                    "packing fraction 0.1-0.3, 16 replicas" % n_systems)


def assembly(seed: int = 0, mc_steps: int = 10_000) -> Workload:
    rng = np.random.default_rng(seed)
    table = contact_table(rng)
    chain = compact_chain(rng, 150)
    types = rng.integers(0, 20, size=150)
    s = build_system(rng, table, [(types, chain)] * 60, 2000, 10.0, 400.0)
    R = 32
    return Workload("assembly", [s], [R], [geometric_ladder(290.0, 500.0, R)], 0.5, 0.2,
                    benchmark_params(), mc_steps, 1000,
                    "60 x 150-residue chains + 2000 crowders R=10 A, 400 A box, 32 replicas")


WORKLOADS = {"two_chain": two_chain, "crowded": crowded, "batch64": batch64,
             "assembly": assembly}


def write_reference_inputs(workload: Workload, system_index: int, directory: str,
                           mc_steps: int, resteps: int, threads: int,
                           sample_frequency: Optional[int] = None) -> str:
    """Write one system of a workload in the reference's own input formats:
    data/AminoAcids, data/pair_potentials_MJ1996 (the file name the reference
    reads, holding this workload's raw table), one CA-only PDB per chain and
    per crowder, and a config file with 'p(x,y,z) r(...)' placement lines.
    Returns the config path. The reference applies its own compile-time
    lambda (0.159) and crowder model ((6/r)^6, 15 A cutoff)."""
    s = workload.systems[system_index]
    R = workload.n_replicas[system_index]
    os.makedirs(os.path.join(directory, "data"), exist_ok=True)
    os.makedirs(os.path.join(directory, "pdb"), exist_ok=True)
    s.table.write(os.path.join(directory, "data", "AminoAcids"))
    s.table.write_pairs(os.path.join(directory, "data", "pair_potentials_MJ1996"))
    lad = workload.ladders[system_index]
    lines = ["gpus 1", "streams 1", "threads %d" % min(threads, R), "mcsteps %d" % mc_steps,
             "resteps %d" % resteps, "replicas %d" % R,
             "samplefrequency %d" % (sample_frequency or max(1, mc_steps // resteps)),
             "sampleafter %d" % mc_steps, "boundry %r" % float(s.box),
             "temperaturemax %r" % float(lad[-1]), "temperaturemin %r" % float(lad[0]),
             "prefix synth", "files"]
    crowder_pdb = os.path.join(directory, "pdb", "crowder.pdb")
    write_pdb_ca(crowder_pdb, [0], np.zeros((1, 3), np.float32), s.table)
    for i, m in enumerate(s.molecules):
        if m.crowder:
            continue
        path = os.path.join(directory, "pdb", "chain%03d.pdb" % i)
        # the chain in its current frame: rel coordinates, placed at its centre
        write_pdb_ca(path, m.types, m.rel, s.table, chain="A")
        lines.append("p(%r,%r,%r) r(0,0,1,-1) %s" % (float(m.centre[0]), float(m.centre[1]),
                                                      float(m.centre[2]), path))
    lines.append("crowders")
    for m in s.molecules:
        if m.crowder:
            lines.append("p(%r,%r,%r) r(0,0,1,-1) %s" % (float(m.centre[0]), float(m.centre[1]),
                                                          float(m.centre[2]), crowder_pdb))
    cfg = os.path.join(directory, "config")
    with open(cfg, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return cfg
