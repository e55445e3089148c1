"""Host-side system model: residue tables, rigid molecules, systems.

Mirrors the reference's host classes and file formats so that a system built
here holds bit-identical FP32 coordinates to the one the reference builds:

  AminoAcidTable.load ....... AminoAcids::loadAminoAcidData
                              (simulation engine/src/AminoAcids.cpp:25-71)
  AminoAcidTable.load_pairs . AminoAcids::loadLJPotentialData (AminoAcids.cpp:73-139)
  Molecule.from_pdb ......... Molecule::initFromPDB, CA beads only (Molecule.cpp:430-830)
  Molecule.translate ........ Molecule::translate (Molecule.cpp:146-171)
  Molecule.set_position ..... Molecule::setPosition (Molecule.cpp:247-260)
  Molecule.rotate_q ......... Molecule::rotateQ + Quaternion::rotateVector
                              (Molecule.cpp:288-333, Quaternion.cpp:84-101)

FP32 quantities are numpy.float32 scalars (IEEE single rounding per operation,
as the reference's float arithmetic on x86-64 without FMA); FP64 quantities are
Python floats.
"""
from __future__ import annotations

import dataclasses
import math
import re
import os
from typing import Iterable, List, Optional, Sequence

import numpy as np

from ._capi import MAX_TYPES, NUM_AMINO

f32 = np.float32

# ------------------------------------------------------------------ constants
# simulation engine/src/definitions.h:11-35, 84-93 (float literals)
RGAS = f32(8.314472)
KBT_CONVERSION_FACTOR = f32(f32(1.0) / (f32(f32(294.0) * RGAS) / f32(4184.0)))
LJ_CONVERSION_FACTOR = f32(0.3507221006079)
DH_CONSTANT = f32(f32(f32(0.948) * f32(1.602176487)) * f32(1.602176487))  # Replica.cpp:624
LAMBDA_MJ1996 = f32(0.159)
E0_MJ1996 = f32(-2.27)
DEBYE_LENGTH = f32(10.0)
CROWDER_CUTOFF = f32(15.0)
BOUND_ENERGY = f32(-1.1844)  # definitions.h:84
CROWDER_TYPE = NUM_AMINO      # first crowder species type index

# The 20 standard residues; the default table order follows the reference's
# data/AminoAcids file (one-letter codes A R N D C E Q G L K M F P S T W Y V H I).
STANDARD_RESIDUES = [
    ("Alanine", "Ala", "A"), ("Arginine", "Arg", "R"), ("Asparagine", "Asn", "N"),
    ("Aspartic_acid", "Asp", "D"), ("Cysteine", "Cys", "C"), ("Glutamic_acid", "Glu", "E"),
    ("Glutamine", "Gln", "Q"), ("Glycine", "Gly", "G"), ("Leucine", "Leu", "L"),
    ("Lysine", "Lys", "K"), ("Methionine", "Met", "M"), ("Phenylalanine", "Phe", "F"),
    ("Proline", "Pro", "P"), ("Serine", "Ser", "S"), ("Threonine", "Thr", "T"),
    ("Tryptophan", "Trp", "W"), ("Tyrosine", "Tyr", "Y"), ("Valine", "Val", "V"),
    ("Histidine", "His", "H"), ("Isoleucine", "Ile", "I"),
]


class ModelError(ValueError):
    pass


# ------------------------------------------------------------------ residue table
@dataclasses.dataclass
class AminoAcidTable:
    """20 residue types (name, 3-letter name, symbol, vdW radius, charge) and the
    raw 20x20 contact table M_ab (eps_ab = lambda (M_ab - e0))."""

    names: List[str]
    snames: List[str]
    symbols: List[str]
    vdw: np.ndarray      # float32[20]
    charge: np.ndarray   # float32[20]
    pairs: np.ndarray    # float32[20, 20]

    @staticmethod
    def load(path: str) -> "AminoAcidTable":
        """Parse the reference's data/AminoAcids format: blocks of five lines
        (name, abbreviation, symbol, vdW radius, charge); '#' lines and blank
        lines are skipped (AminoAcids.cpp:25-71)."""
        with open(path, "r", errors="replace") as fh:
            lines = [ln.rstrip("\r\n") for ln in fh]
        names, snames, symbols, vdw, charge = [], [], [], [], []
        i = 0
        while i < len(lines) and len(names) < 20:
            ln = lines[i]
            if ln == "" or ln.startswith("#"):
                i += 1
                continue
            if i + 4 >= len(lines):
                raise ModelError("%s: truncated residue block at line %d" % (path, i + 1))
            names.append(ln[:19])
            snames.append(lines[i + 1][:3])
            symbols.append(lines[i + 2][:1])
            vdw.append(_atof(lines[i + 3]))
            charge.append(_scanf_float(lines[i + 4]))
            i += 5
        if len(names) != 20:
            raise ModelError("%s: expected 20 residue types, found %d" % (path, len(names)))
        return AminoAcidTable(names, snames, symbols, np.array(vdw, np.float32),
                              np.array(charge, np.float32), np.zeros((20, 20), np.float32))

    def index(self, name: str) -> int:
        """AminoAcids::getAminoAcidIndex (AminoAcids.cpp:146-182): 3-letter
        names match case-insensitively on the first letter upper, rest lower;
        1-letter names match the symbol; otherwise the full name."""
        if len(name) < 1:
            return -1
        if len(name) == 3:
            key = name[0].upper() + name[1].lower() + name[2].lower()
            for i in range(19, -1, -1):
                if self.snames[i] == key:
                    return i
        elif len(name) == 1:
            key = name[0].upper()
            for i in range(19, -1, -1):
                if self.symbols[i] == key:
                    return i
        else:
            key = name[0].upper() + name[1:]
            for i in range(19, -1, -1):
                if self.names[i] == key:
                    return i
        return -1

    def load_pairs(self, path: str) -> None:
        """Parse a reference pair-potential file: a label row then an upper
        triangle, mirrored (AminoAcids.cpp:73-139)."""
        with open(path, "r", errors="replace") as fh:
            lines = [ln.rstrip("\r\n") for ln in fh]
        labels: List[int] = []
        start = 0
        M = np.zeros((20, 20), np.float32)
        for ln in lines:
            if ln == "" or ln.startswith("#"):
                continue
            toks = ln.split()
            if not labels:
                labels = [self.index(t) for t in toks]
                if len(labels) != 20 or min(labels) < 0:
                    raise ModelError("%s: bad label row" % path)
                continue
            vals = toks[1:]
            if start >= 20:
                break
            if len(vals) < 20 - start:
                raise ModelError("%s: row %d too short" % (path, start + 1))
            for j in range(start, 20):
                v = _scanf_float(vals[j - start])
                M[labels[start], labels[j]] = v
                M[labels[j], labels[start]] = v
            start += 1
        if start != 20:
            raise ModelError("%s: expected 20 rows, found %d" % (path, start))
        self.pairs = M

    @staticmethod
    def synthetic(vdw: float = 6.0, his_charge: float = 0.0) -> "AminoAcidTable":
        """Uniform radii, K/R +1, D/E -1, others 0 (His configurable)."""
        names = [r[0] for r in STANDARD_RESIDUES]
        snames = [r[1] for r in STANDARD_RESIDUES]
        symbols = [r[2] for r in STANDARD_RESIDUES]
        q = np.zeros(20, np.float32)
        for i, s in enumerate(symbols):
            if s in ("K", "R"):
                q[i] = 1.0
            elif s in ("D", "E"):
                q[i] = -1.0
            elif s == "H":
                q[i] = his_charge
        return AminoAcidTable(names, snames, symbols, np.full(20, vdw, np.float32), q,
                              np.zeros((20, 20), np.float32))

    def write(self, path: str) -> None:
        """Write in the reference's data/AminoAcids format."""
        with open(path, "w") as fh:
            for i in range(20):
                fh.write("#Amino acid class initialisation data\n#name\n#abbriviation\n"
                         "#short symbol\n#van der Waal radius\n#residue charge\n")
                fh.write("%s\n%s\n%s\n%s\n%s\n\n\n" % (self.names[i], self.snames[i],
                                                         self.symbols[i], _fmt(self.vdw[i]),
                                                         _fmt(self.charge[i])))

    def write_pairs(self, path: str) -> None:
        """Write the raw table in the reference's pair-potential format."""
        with open(path, "w") as fh:
            fh.write("# raw contact table M_ab (eps_ab = lambda (M_ab - e0))\n")
            fh.write("     " + " ".join("%s" % s for s in self.snames) + "\n")
            for i in range(20):
                # shortest FP32 round-trip text: the reference reads rows into a
                # 255-character buffer (AminoAcids.cpp:104)
                fh.write(self.snames[i] + " " +
                         " ".join(_f32_text(self.pairs[i, j]) for j in range(i, 20)) + "\n")


def _fmt(v) -> str:
    return _f32_text(v)


def _f32_text(v) -> str:
    """Shortest decimal text that reads back as the same float32."""
    return str(np.float32(v))


def _atof(s: str) -> float:
    import re
    m = re.match(r"\s*[-+]?(\d+\.?\d*|\.\d+)([eE][-+]?\d+)?", s)
    return float(m.group(0)) if m else 0.0


def _scanf_float(s: str) -> float:
    return float(np.float32(_atof(s)))


# ------------------------------------------------------------------ molecules
@dataclasses.dataclass
class Molecule:
    """A rigid molecule: bead types, absolute positions, positions relative to
    the centre, centre and accumulated rotation quaternion (w, x, y, z)."""

    types: np.ndarray      # int32[n]
    pos: np.ndarray        # float32[n, 3]
    rel: np.ndarray        # float32[n, 3]
    centre: np.ndarray     # float32[3]
    quat: np.ndarray       # float64[4]
    crowder: bool = False
    name: str = ""
    res_seq: Optional[np.ndarray] = None  # PDB residue numbers (Residue::resSeq)
    radius: Optional[float] = None  # a crowder's own radius (else the system's)

    @property
    def n(self) -> int:
        return int(self.types.shape[0])

    @staticmethod
    def from_beads(types: Sequence[int], pos: np.ndarray, name: str = "") -> "Molecule":
        """Centre = FP32 running sum / count, rel = pos - centre
        (Molecule.cpp:800-818)."""
        pos = np.asarray(pos, np.float32).reshape(-1, 3)
        n = pos.shape[0]
        if n == 0:
            raise ModelError("molecule %s has no CA beads" % name)
        c = [f32(0.0), f32(0.0), f32(0.0)]
        for i in range(n):
            for k in range(3):
                c[k] = f32(c[k] + pos[i, k])
        nf = f32(n)
        centre = np.array([f32(c[0] / nf), f32(c[1] / nf), f32(c[2] / nf)], np.float32)
        rel = (pos - centre[None, :]).astype(np.float32)
        return Molecule(np.asarray(types, np.int32).copy(), pos.copy(), rel, centre,
                        np.array([1.0, 0.0, 0.0, 0.0]), False, name)

    @staticmethod
    def from_pdb(path: str, table: AminoAcidTable) -> "Molecule":
        types, xyz, seq = read_pdb_ca(path, table, with_seq=True)
        m = Molecule.from_beads(types, xyz, name=path)
        m.res_seq = seq
        return m

    def copy(self) -> "Molecule":
        return Molecule(self.types.copy(), self.pos.copy(), self.rel.copy(), self.centre.copy(),
                        self.quat.copy(), self.crowder, self.name,
                        None if self.res_seq is None else self.res_seq.copy(), self.radius)

    def translate(self, v) -> None:
        """Molecule::translate: centre and every bead += v (FP32)."""
        v = np.asarray(v, np.float32)
        self.centre = (self.centre + v).astype(np.float32)
        self.pos = (self.pos + v[None, :]).astype(np.float32)

    def set_position(self, v) -> None:
        """Molecule::setPosition: centre = v, bead = rel + centre (FP32)."""
        self.centre = np.asarray(v, np.float32).copy()
        self.pos = (self.rel + self.centre[None, :]).astype(np.float32)

    def rotate_q(self, axis, angle: float) -> None:
        """Molecule::rotateQ (axis already normalised, FP64)."""
        sina = math.sin(angle / 2.0)
        cosa = math.cos(angle / 2.0)
        qw, qx, qy, qz = cosa, sina * axis[0], sina * axis[1], sina * axis[2]
        mag = math.sqrt(qw * qw + qx * qx + qy * qy + qz * qz)
        qw, qx, qy, qz = qw / mag, qx / mag, qy / mag, qz / mag
        r = self.quat
        self.quat = np.array([
            qw * r[0] - qx * r[1] - qy * r[2] - qz * r[3],
            qw * r[1] + qx * r[0] + qy * r[3] - qz * r[2],
            qw * r[2] - qx * r[3] + qy * r[0] + qz * r[1],
            qw * r[3] + qx * r[2] - qy * r[1] + qz * r[0]])
        self.rel = rotate_vectors(qw, qx, qy, qz, self.rel)
        self.pos = (self.rel + self.centre[None, :]).astype(np.float32)


def rotate_vectors(w: float, x: float, y: float, z: float, v: np.ndarray) -> np.ndarray:
    """Quaternion::rotateVector in FP64 with the reference's operation order,
    each component rounded to FP32 (Quaternion.cpp:84-101)."""
    w2, x2, y2, z2 = w * w, x * x, y * y, z * z
    wx, wy, wz = w * x, w * y, w * z
    xy, xz, yz = x * y, x * z, y * z
    a = w2 + x2 - y2 - z2
    b, c = xy - wz, wy + xz
    d, e = wz + xy, yz - wx
    f = w2 - x2 + y2 - z2
    g, h = xz - wy, yz + wx
    i = w2 - x2 - y2 + z2
    vx = v[:, 0].astype(np.float64)
    vy = v[:, 1].astype(np.float64)
    vz = v[:, 2].astype(np.float64)
    X = vx * a + (vy * b + vz * c) * 2.0
    Y = (vx * d + vz * e) * 2.0 + vy * f
    Z = (vx * g + vy * h) * 2.0 + vz * i
    return np.stack([X, Y, Z], axis=1).astype(np.float32)


def normalise_axis(rx: float, ry: float, rz: float):
    """Vector3double::normalizeInPlace (vector3f.cpp:36-43)."""
    m = math.sqrt(rx * rx + ry * ry + rz * rz)
    return (rx / m, ry / m, rz / m)


# ------------------------------------------------------------------ PDB
def read_pdb_ca(path: str, table: AminoAcidTable, with_seq: bool = False):
    """CA beads of a PDB file, as Molecule::initFromPDB reads them.

    Fixed columns: atom name 13-16, residue name 18-20, x/y/z 31-38/39-46/47-54.
    Reproduces the reference reader's buffer reuse: an empty line (including
    the empty read at end of file after a final newline) re-processes the
    previous line, so a file that ends in an ATOM CA line followed by a newline
    yields that bead twice, as in the reference (its getline buffer is not
    cleared, Molecule.cpp:456-459). Unknown residue names raise ModelError
    (the reference would index its table at -1)."""
    with open(path, "rb") as fh:
        data = fh.read().decode("latin-1")
    raw = data.split("\n")
    # getline semantics: the last element is "" when the file ends in "\n",
    # and that empty read is processed once more before eof stops the loop
    types: List[int] = []
    xyz: List[List[float]] = []
    seq: List[int] = []
    prev = ""
    for ln in raw:
        ln = ln.rstrip("\r")[:511]
        cur = ln if ln != "" else prev
        if ln != "":
            prev = ln
        tok = cur.lstrip(" ").split(" ", 1)[0]  # strtok(line, " ")
        if tok != "ATOM":
            continue
        name = cur[12:16].split()
        if not name or name[0] != "CA":
            continue
        res = cur[17:20].split()
        t = table.index(res[0] if res else "")
        if t < 0:
            raise ModelError("%s: unknown residue name %r" % (path, cur[17:20]))
        x = _scanf_float(cur[30:38])
        y = _scanf_float(cur[38:46])
        z = _scanf_float(cur[46:54])
        types.append(t)
        xyz.append([x, y, z])
        m = re.match(r"\s*[-+]?\d+", cur[22:26])  # resSeq, columns 23-26 (sscanf %d)
        seq.append(int(m.group(0)) if m else 0)
    if not types:
        raise ModelError("%s: no CA atoms" % path)
    if with_seq:
        return np.array(types, np.int32), np.array(xyz, np.float32), np.array(seq, np.int32)
    return np.array(types, np.int32), np.array(xyz, np.float32)


def write_pdb_ca(path: str, types: Sequence[int], xyz: np.ndarray, table: AminoAcidTable,
                 chain: str = "A") -> None:
    with open(path, "w") as fh:
        fh.write("REMARK generated CA-only structure\n")
        for i, (t, p) in enumerate(zip(types, xyz)):
            fh.write("ATOM  %5d  CA  %3s %s%4d    %8.3f%8.3f%8.3f  1.00  1.00\n" %
                     (i + 1, table.snames[int(t)].upper(), chain, i + 1, p[0], p[1], p[2]))
        fh.write("END\n")


# ------------------------------------------------------------------ systems
@dataclasses.dataclass
class System:
    """One REMC system: molecules (chains first, then crowders), box, and the
    type tables shared with the engine."""

    molecules: List[Molecule]
    box: float
    table: AminoAcidTable
    crowder_radius: float = 0.0
    translate_only_crowders: bool = False

    @property
    def n_beads(self) -> int:
        return sum(m.n for m in self.molecules)

    @property
    def n_mol(self) -> int:
        return len(self.molecules)

    @property
    def n_chains(self) -> int:
        return sum(1 for m in self.molecules if not m.crowder)

    def radius_of(self, m: Molecule) -> float:
        return float(self.crowder_radius if m.radius is None else m.radius)

    def crowder_radii(self) -> List[float]:
        """Distinct crowder radii in order of first appearance; crowder
        species k (bead type CROWDER_TYPE + k) has the k-th of them."""
        radii: List[float] = []
        for m in self.molecules:
            if m.crowder and self.radius_of(m) not in radii:
                radii.append(self.radius_of(m))
        if len(radii) > MAX_TYPES - CROWDER_TYPE:
            raise ModelError("at most %d crowder radii per system" % (MAX_TYPES - CROWDER_TYPE))
        return radii

    def topology(self):
        mol_start = np.zeros(self.n_mol + 1, np.int32)
        roles = np.zeros(self.n_mol, np.int32)
        types = []
        radii = self.crowder_radii()
        for i, m in enumerate(self.molecules):
            mol_start[i + 1] = mol_start[i] + m.n
            roles[i] = -1 if m.crowder else 0
            if m.crowder:
                types.append(np.full(m.n, CROWDER_TYPE + radii.index(self.radius_of(m)), np.int32))
            else:
                types.append(m.types)
        return mol_start, roles, np.concatenate(types).astype(np.int32)

    def state(self):
        pos = np.concatenate([m.pos for m in self.molecules]).astype(np.float32)
        rel = np.concatenate([m.rel for m in self.molecules]).astype(np.float32)
        centre = np.stack([m.centre for m in self.molecules]).astype(np.float32)
        quat = np.stack([m.quat for m in self.molecules]).astype(np.float64)
        return pos, rel, centre, quat

    def type_tables(self):
        """(vdw, charge, rho) per engine type: residue types from the table,
        rho = vdW/2 for residues; crowder species 20.. carry their crowder
        radius (the system's radius where no species uses the type)."""
        vdw = np.zeros(MAX_TYPES, np.float32)
        q = np.zeros(MAX_TYPES, np.float32)
        rho = np.zeros(MAX_TYPES, np.float32)
        vdw[:20] = self.table.vdw
        q[:20] = self.table.charge
        rho[:20] = self.table.vdw * np.float32(0.5)
        rho[20:] = np.float32(self.crowder_radius)
        for k, r in enumerate(self.crowder_radii()):
            rho[CROWDER_TYPE + k] = np.float32(r)
        return vdw, q, rho


def geometric_ladder(tmin: float, tmax: float, n: int) -> np.ndarray:
    """REMCSimulation's ladder (main.cpp:1161-1169):
    T_i = Tmin * pow(double(Tmax/Tmin) ^ (1/(n-1)), i), stored as float."""
    tmin32, tmax32 = f32(tmin), f32(tmax)
    if n == 1:
        return np.array([tmin32], np.float32)
    g = math.pow(float(f32(tmax32 / tmin32)), 1.0 / float(n - 1))
    return np.array([f32(float(tmin32) * math.pow(g, i)) for i in range(n)], np.float32)


def reference_step_ladder(n: int):
    """Per-replica translate (0.5..5 A) and rotate (0.1..0.5 rad) steps of the
    reference driver (main.cpp:1163-1178, definitions.h:78-83)."""
    if n == 1:
        return np.array([0.5], np.float32), np.array([float(f32(0.1))])
    # MAX/MIN are float literals divided in FP32, then widened
    gt = math.pow(float(f32(f32(5.0) / f32(0.5))), 1.0 / float(n - 1))
    gr = math.pow(float(f32(f32(0.5) / f32(0.1))), 1.0 / float(n - 1))
    tr = np.array([f32(float(f32(0.5)) * math.pow(gt, i)) for i in range(n)], np.float32)
    # setRotateStep takes a double; MIN_ROTATION is a float literal
    ro = np.array([float(f32(0.1)) * math.pow(gr, i) for i in range(n)], np.float64)
    return tr, ro
