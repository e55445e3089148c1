"""ctypes bindings of the two oracles (TEST INFRASTRUCTURE ONLY).

`FP64Oracle` wraps oracle/_build/libremc_oracle.so (remc_oracle.c).
`ReferenceReplica` wraps oracle/_ref/libremcref.so: the reference engine's own
Replica/Molecule sources plus ref_harness.cpp.
Both take systems in the engine's layout (remcdockingsimulator_b200.model.System).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libremc_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libremcref.so")
REF_EXE = os.path.join(HERE, "_ref", "REMCDockingCPU")

PF = C.POINTER(C.c_float)
PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int)


class OracleParams(C.Structure):
    _fields_ = [("lambda_", C.c_float), ("e0", C.c_float), ("debye_length", C.c_float),
                ("dh_const", C.c_float), ("lj_cf", C.c_float), ("kbt_cf", C.c_float),
                ("crowder_mode", C.c_int), ("crowder_cutoff", C.c_float),
                ("crowder_eps", C.c_float)]


class OracleSystem(C.Structure):
    _fields_ = [("n_beads", C.c_int), ("n_mol", C.c_int), ("mol_start", PI), ("mol_role", PI),
                ("bead_type", PI), ("type_vdw", PF), ("type_q", PF), ("type_rho", PF),
                ("eps_table", PF), ("box", C.c_float)]


class OracleReplica(C.Structure):
    _fields_ = [("pos", PF), ("rel", PF), ("centre", PF), ("quat", PD), ("energy", C.c_double),
                ("temperature", C.c_float), ("translate_step", C.c_float),
                ("rotate_cos_half", C.c_double), ("rotate_sin_half", C.c_double),
                ("translate_only_crowders", C.c_int), ("accept", C.c_int),
                ("acceptA", C.c_int), ("reject", C.c_int)]


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


_olib = None
_rlib = None


def oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_LIB):
            from . import build
            build.build_oracle()
        L = C.CDLL(ORACLE_LIB)
        L.oracle_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                           C.POINTER(C.c_uint32)]
        L.oracle_step_uniforms.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, PD]
        L.oracle_exchange_uniform.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
        L.oracle_exchange_uniform.restype = C.c_double
        L.oracle_energy_full.argtypes = [C.POINTER(OracleSystem), C.POINTER(OracleParams), PF]
        L.oracle_energy_full.restype = C.c_double
        L.oracle_energy_molecule.argtypes = [C.POINTER(OracleSystem), C.POINTER(OracleParams),
                                             PF, C.c_int, PF]
        L.oracle_energy_molecule.restype = C.c_double
        L.oracle_energy_molecule_abs.argtypes = [C.POINTER(OracleSystem), C.POINTER(OracleParams),
                                                 PF, C.c_int, PF]
        L.oracle_energy_molecule_abs.restype = C.c_double
        L.oracle_noncrowder_pair_energy.argtypes = [C.POINTER(OracleSystem),
                                                    C.POINTER(OracleParams), PF]
        L.oracle_noncrowder_pair_energy.restype = C.c_double
        L.oracle_mc_run.argtypes = [C.POINTER(OracleSystem), C.POINTER(OracleParams),
                                    C.POINTER(OracleReplica), C.c_uint64, C.c_uint32,
                                    C.c_uint32, C.c_uint32, C.c_int, C.c_int, PI, PI, PD]
        L.oracle_exchange_round.argtypes = [C.c_int, C.c_int, PF, PD, PI, PI, C.c_uint64,
                                            C.c_uint32, C.c_uint32, PI]
        L.oracle_exchange_round.restype = C.c_int
        L.oracle_post_rebuild.argtypes = [PF, PI, C.c_int, PI, PF, C.c_float, PD, PF, PF]
        L.oracle_post_drms.argtypes = [PF, PF, PI, C.c_int, C.c_int, C.c_float, C.c_float,
                                       C.POINTER(C.c_longlong)]
        L.oracle_post_drms.restype = C.c_double
        L.oracle_energy_adjoint.argtypes = [C.POINTER(OracleSystem), C.POINTER(OracleParams),
                                            PF, PF, PD, PD, PD, PD]
        _olib = L
    return _olib


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    oracle_lib().oracle_philox4x32_10(c, k, o)
    return list(o)


def step_uniforms(seed: int, step: int, slot: int, system: int) -> np.ndarray:
    u = np.zeros(6)
    oracle_lib().oracle_step_uniforms(seed, step, slot, system, _p(u, C.c_double))
    return u


def exchange_uniform(seed: int, round_: int, pair: int, system: int) -> float:
    return oracle_lib().oracle_exchange_uniform(seed, round_, pair, system)


def post_rebuild(rel0, mol_start, shift, centre0, box, quat, centre):
    """pdbgen's pose reconstruction of one frame (oracle_post_rebuild)."""
    rel0 = np.ascontiguousarray(rel0, np.float32)
    ms = np.ascontiguousarray(mol_start, np.int32)
    sh = np.ascontiguousarray(shift, np.int32)
    c0 = np.ascontiguousarray(centre0, np.float32)
    q = np.ascontiguousarray(quat, np.float64)
    c = np.ascontiguousarray(centre, np.float32)
    pos = np.zeros((int(ms[-1]), 3), np.float32)
    oracle_lib().oracle_post_rebuild(_p(rel0, C.c_float), _p(ms, C.c_int), len(ms) - 1,
                                     _p(sh, C.c_int), _p(c0, C.c_float), box, _p(q, C.c_double),
                                     _p(c, C.c_float), _p(pos, C.c_float))
    return pos


def post_drms(sim, ref, mol_start, reverse=False, native_cut=12.0, recovered_cut=15.0):
    """DRMS of one frame and its (native, recovered, binding) contact counts."""
    x = np.ascontiguousarray(sim, np.float32)
    r = np.ascontiguousarray(ref, np.float32)
    ms = np.ascontiguousarray(mol_start, np.int32)
    cnt = np.zeros(3, np.int64)
    d = oracle_lib().oracle_post_drms(_p(x, C.c_float), _p(r, C.c_float), _p(ms, C.c_int),
                                      len(ms) - 1, 1 if reverse else 0, native_cut, recovered_cut,
                                      cnt.ctypes.data_as(C.POINTER(C.c_longlong)))
    return d, cnt


def params_from(p) -> OracleParams:
    """Copy an engine remc_params (or any object with the same fields)."""
    o = OracleParams()
    for name, _ in OracleParams._fields_:
        setattr(o, name, getattr(p, name))
    return o


class FP64Oracle:
    """The FP64 restatement on one system's topology and tables."""

    def __init__(self, system, params, crowder_type_rho: Optional[dict] = None):
        from remcdockingsimulator_b200._capi import MAX_TYPES
        self.system = system
        self.params = params_from(params)
        mol_start, roles, types = system.topology()
        self.mol_start = np.ascontiguousarray(mol_start, np.int32)
        self.roles = np.ascontiguousarray(roles, np.int32)
        self.types = np.ascontiguousarray(types, np.int32)
        vdw, q, rho = system.type_tables()
        self.vdw = np.ascontiguousarray(vdw, np.float32)
        self.q = np.ascontiguousarray(q, np.float32)
        self.rho = np.ascontiguousarray(rho, np.float32)
        eps = np.zeros((32, 32), np.float32)
        lam = np.float32(self.params.lambda_)
        e0 = np.float32(self.params.e0)
        eps[:20, :20] = lam * (system.table.pairs.astype(np.float32) - e0)  # FP32, as the engine
        self.eps = np.ascontiguousarray(eps.reshape(-1), np.float32)
        self.raw = np.ascontiguousarray(system.table.pairs.reshape(-1), np.float32)
        s = OracleSystem()
        s.n_beads = system.n_beads
        s.n_mol = system.n_mol
        s.mol_start = _p(self.mol_start, C.c_int)
        s.mol_role = _p(self.roles, C.c_int)
        s.bead_type = _p(self.types, C.c_int)
        s.type_vdw = _p(self.vdw, C.c_float)
        s.type_q = _p(self.q, C.c_float)
        s.type_rho = _p(self.rho, C.c_float)
        s.eps_table = _p(self.eps, C.c_float)
        s.box = system.box
        self.s = s

    def energy(self, pos: np.ndarray) -> float:
        pos = np.ascontiguousarray(pos, np.float32)
        return oracle_lib().oracle_energy_full(C.byref(self.s), C.byref(self.params),
                                               _p(pos, C.c_float))

    def energy_molecule(self, pos: np.ndarray, m: int, mpos: np.ndarray) -> float:
        pos = np.ascontiguousarray(pos, np.float32)
        mpos = np.ascontiguousarray(mpos, np.float32)
        return oracle_lib().oracle_energy_molecule(C.byref(self.s), C.byref(self.params),
                                                   _p(pos, C.c_float), m, _p(mpos, C.c_float))

    def energy_molecule_abs(self, pos: np.ndarray, m: int, mpos: np.ndarray) -> float:
        """Sum of |pair term| of molecule m placed at mpos against the rest."""
        pos = np.ascontiguousarray(pos, np.float32)
        mpos = np.ascontiguousarray(mpos, np.float32)
        return oracle_lib().oracle_energy_molecule_abs(C.byref(self.s), C.byref(self.params),
                                                       _p(pos, C.c_float), m, _p(mpos, C.c_float))

    def noncrowder_pair_energy(self, pos: np.ndarray) -> float:
        pos = np.ascontiguousarray(pos, np.float32)
        return oracle_lib().oracle_noncrowder_pair_energy(C.byref(self.s), C.byref(self.params),
                                                          _p(pos, C.c_float))

    def adjoint(self, pos: np.ndarray):
        pos = np.ascontiguousarray(pos, np.float32)
        f = np.zeros((self.system.n_beads, 3))
        dl = C.c_double()
        dx = C.c_double()
        de = np.zeros(32 * 32)
        oracle_lib().oracle_energy_adjoint(C.byref(self.s), C.byref(self.params),
                                           _p(pos, C.c_float), _p(self.raw, C.c_float),
                                           _p(f, C.c_double), C.byref(dl), C.byref(dx),
                                           _p(de, C.c_double))
        return f, dl.value, dx.value, de.reshape(32, 32)

    def mc_run(self, state, temperature: float, translate_step: float, rotate_step: float,
               seed: int, step0: int, slot: int, system_index: int, n_steps: int,
               energy: float, energy_mode: int = 0):
        """Run n_steps on a copy of `state` (pos, rel, centre, quat); returns
        (new state, energy, flags, molecules, dE, counters)."""
        import math
        pos, rel, cen, quat = [np.ascontiguousarray(a).copy() for a in state]
        pos = np.ascontiguousarray(pos, np.float32)
        rel = np.ascontiguousarray(rel, np.float32)
        cen = np.ascontiguousarray(cen, np.float32)
        quat = np.ascontiguousarray(quat, np.float64)
        r = OracleReplica()
        r.pos = _p(pos, C.c_float)
        r.rel = _p(rel, C.c_float)
        r.centre = _p(cen, C.c_float)
        r.quat = _p(quat, C.c_double)
        r.energy = energy
        r.temperature = temperature
        r.translate_step = translate_step
        r.rotate_cos_half = math.cos(rotate_step / 2.0)
        r.rotate_sin_half = math.sin(rotate_step / 2.0)
        r.translate_only_crowders = 1 if self.system.translate_only_crowders else 0
        flags = np.zeros(n_steps, np.int32)
        mol = np.zeros(n_steps, np.int32)
        dE = np.zeros(n_steps)
        oracle_lib().oracle_mc_run(C.byref(self.s), C.byref(self.params), C.byref(r), seed,
                                   step0, slot, system_index, n_steps, energy_mode,
                                   _p(flags, C.c_int), _p(mol, C.c_int), _p(dE, C.c_double))
        return ((pos, rel, cen, quat), r.energy, flags, mol, dE,
                (r.accept, r.acceptA, r.reject))


def exchange_round(ladder, energies, temp_of_slot, slot_of_temp, offset, seed, round_, system):
    lad = np.ascontiguousarray(ladder, np.float32)
    en = np.ascontiguousarray(energies, np.float64)
    tos = np.ascontiguousarray(temp_of_slot, np.int32).copy()
    sot = np.ascontiguousarray(slot_of_temp, np.int32).copy()
    R = lad.size
    acc = np.zeros(max(1, R // 2 + 1), np.int32)
    n = oracle_lib().oracle_exchange_round(R, offset, _p(lad, C.c_float), _p(en, C.c_double),
                                           _p(tos, C.c_int), _p(sot, C.c_int), seed, round_,
                                           system, _p(acc, C.c_int))
    return n, tos, sot, acc


# ---------------------------------------------------------------- reference
def ref_lib():
    global _rlib
    if _rlib is None:
        if not os.path.exists(REF_LIB):
            from . import build
            if not build.build_reference():
                raise RuntimeError("reference harness not built and the reference tree is absent")
        L = C.CDLL(REF_LIB)
        L.ref_replica_create.argtypes = [PF, PF, PF, C.c_int, PI, PI, PI, PF, PF, PF, PD,
                                         C.c_float, C.c_float]
        L.ref_replica_create.restype = C.c_void_p
        L.ref_replica_destroy.argtypes = [C.c_void_p]
        L.ref_replica_E.argtypes = [C.c_void_p]
        L.ref_replica_E.restype = C.c_double
        L.ref_replica_E_pair.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.ref_replica_E_pair.restype = C.c_float
        L.ref_replica_potential.argtypes = [C.c_void_p]
        L.ref_replica_potential.restype = C.c_double
        L.ref_replica_set_steps.argtypes = [C.c_void_p, C.c_float, C.c_double]
        L.ref_replica_get_state.argtypes = [C.c_void_p, PF, PF, PF, PD]
        L.ref_replica_mcsearch.argtypes = [C.c_void_p, C.c_int, PD, PI, PI, PD]
        L.ref_replica_mcsearch.restype = C.c_int
        L.ref_random_vectors.argtypes = [C.c_void_p, PD, PF, PD]
        L.ref_time_mcsearch.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int]
        L.ref_time_mcsearch.restype = C.c_double
        L.ref_run_mcsearch.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int]
        L.ref_run_mcsearch.restype = C.c_double
        L.ref_replica_seed.argtypes = [C.c_void_p, C.c_uint]
        L.ref_replica_counters.argtypes = [C.c_void_p, PI]
        _rlib = L
    return _rlib


def reference_available() -> bool:
    try:
        ref_lib()
        return True
    except Exception:
        return False


class ReferenceReplica:
    """The reference's own Replica built from a system's state (crowders use the
    reference's (6/r)^6 model with its 15 A cutoff and lambda = 0.159)."""

    def __init__(self, system, state=None, temperature: float = 300.0):
        self.system = system
        mol_start, roles, types = system.topology()
        self.n_beads = system.n_beads
        self.n_mol = system.n_mol
        # the reference keeps the residue's own type index for crowder beads'
        # charge/radius lookup; crowders carry type 0 here (unused by (6/r)^6)
        rt = np.where(types >= 20, 0, types).astype(np.int32)
        pos, rel, cen, quat = state if state is not None else system.state()
        self._keep = [np.ascontiguousarray(a) for a in (
            system.table.vdw.astype(np.float32), system.table.charge.astype(np.float32),
            system.table.pairs.astype(np.float32).reshape(-1), mol_start.astype(np.int32),
            roles.astype(np.int32), rt, np.asarray(pos, np.float32).reshape(-1),
            np.asarray(rel, np.float32).reshape(-1), np.asarray(cen, np.float32).reshape(-1),
            np.asarray(quat, np.float64).reshape(-1))]
        k = self._keep
        self.h = ref_lib().ref_replica_create(
            _p(k[0], C.c_float), _p(k[1], C.c_float), _p(k[2], C.c_float), self.n_mol,
            _p(k[3], C.c_int), _p(k[4], C.c_int), _p(k[5], C.c_int), _p(k[6], C.c_float),
            _p(k[7], C.c_float), _p(k[8], C.c_float), _p(k[9], C.c_double), system.box,
            temperature)

    def close(self):
        if self.h:
            ref_lib().ref_replica_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def E(self) -> float:
        return ref_lib().ref_replica_E(self.h)

    def E_pair(self, a: int, b: int) -> float:
        return ref_lib().ref_replica_E_pair(self.h, a, b)

    @property
    def potential(self) -> float:
        return ref_lib().ref_replica_potential(self.h)

    def set_steps(self, translate_step: float, rotate_step: float) -> None:
        ref_lib().ref_replica_set_steps(self.h, translate_step, rotate_step)

    def state(self):
        pos = np.zeros((self.n_beads, 3), np.float32)
        rel = np.zeros((self.n_beads, 3), np.float32)
        cen = np.zeros((self.n_mol, 3), np.float32)
        quat = np.zeros((self.n_mol, 4))
        ref_lib().ref_replica_get_state(self.h, _p(pos, C.c_float), _p(rel, C.c_float),
                                        _p(cen, C.c_float), _p(quat, C.c_double))
        return pos, rel, cen, quat

    def steps_set(self, translate_step: float, rotate_step: float) -> None:
        self.set_steps(translate_step, rotate_step)

    def seed(self, seed: int) -> None:
        """Leave fed mode; seed the replica's own MT19937 generators."""
        ref_lib().ref_replica_seed(self.h, seed)

    def counters(self):
        out = np.zeros(3, np.int32)
        ref_lib().ref_replica_counters(self.h, _p(out, C.c_int))
        return tuple(int(x) for x in out)

    def mcsearch(self, u: np.ndarray):
        """Run len(u) reference MCSearch steps fed with u[s] = 6 uniforms."""
        u = np.ascontiguousarray(u, np.float64).reshape(-1, 6)
        n = u.shape[0]
        flags = np.zeros(n, np.int32)
        mol = np.zeros(n, np.int32)
        en = np.zeros(n)
        under = ref_lib().ref_replica_mcsearch(self.h, n, _p(u, C.c_double), _p(flags, C.c_int),
                                               _p(mol, C.c_int), _p(en, C.c_double))
        return flags, mol, en, under


def run_reference_mcsearch(replicas, n_threads: int, n_steps: int) -> float:
    """The reference's own MCSearch(n_steps) with its own generators (seed
    them first with ReferenceReplica.seed) on every replica, spread over
    n_threads host threads; returns wall seconds."""
    arr = (C.c_void_p * len(replicas))(*[r.h for r in replicas])
    return ref_lib().ref_run_mcsearch(arr, len(replicas), n_threads, n_steps)


def time_reference_mcsearch(replicas, n_threads: int, n_steps: int) -> float:
    """Wall seconds of the reference's own MCSearch(n_steps) on every replica,
    spread over n_threads host threads."""
    arr = (C.c_void_p * len(replicas))(*[r.h for r in replicas])
    return ref_lib().ref_time_mcsearch(arr, len(replicas), n_threads, n_steps)
