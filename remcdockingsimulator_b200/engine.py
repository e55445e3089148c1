"""Python mirror of the engine handle (include/remc_b200.h).

`Engine` owns one remc handle: many independent systems, each with its own
replicas, resident on one GPU. It is the layer the tests and bench drive; the
C++ facade (csrc/remc_replica.h) offers the same operations under the
reference's Replica/Molecule names.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _capi
from ._capi import (MAX_TYPES, NUM_AMINO, Params, SamplePose, SampleRecord, SystemDesc, check,
                    lib)
from .model import System


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def reference_params() -> Params:
    """The reference's compile-time energy constants (definitions.h:11-35,
    Replica.cpp:624), built without loading the engine library: the same
    FP32 values remc_default_params writes (a CPU test compares the two)."""
    from .model import DH_CONSTANT, KBT_CONVERSION_FACTOR, LJ_CONVERSION_FACTOR
    p = Params()
    p.lambda_ = 0.159
    p.e0 = -2.27
    p.debye_length = 10.0
    p.dh_const = float(DH_CONSTANT)
    p.lj_cf = float(LJ_CONVERSION_FACTOR)
    p.kbt_cf = float(KBT_CONVERSION_FACTOR)
    p.crowder_mode = 0
    p.crowder_cutoff = 15.0
    p.crowder_eps = 1.0
    return p


def make_params(lambda_: float = 0.159, e0: float = -2.27, debye_length: float = 10.0,
                crowder_mode: int = 0, crowder_cutoff: float = 15.0,
                crowder_eps: float = 1.0) -> Params:
    p = reference_params()
    p.lambda_ = lambda_
    p.e0 = e0
    p.debye_length = debye_length
    p.crowder_mode = crowder_mode
    p.crowder_cutoff = crowder_cutoff
    p.crowder_eps = crowder_eps
    return p


class Engine:
    """All replicas of all `systems` on one GPU.

    systems[s] is replicated n_replicas[s] times (every replica starts from the
    system's coordinates unless `upload_state` is called with per-instance
    arrays). Instances are numbered system-major, slot-minor."""

    def __init__(self, systems: Sequence[System], n_replicas, params: Optional[Params] = None):
        if isinstance(n_replicas, int):
            n_replicas = [n_replicas] * len(systems)
        if len(n_replicas) != len(systems):
            raise ValueError("one replica count per system")
        self.systems = list(systems)
        self.n_replicas = [int(r) for r in n_replicas]
        self.params = params if params is not None else make_params()
        table0 = self.systems[0].table
        for s in self.systems[1:]:
            if not (np.array_equal(s.table.vdw, table0.vdw) and
                    np.array_equal(s.table.charge, table0.charge) and
                    np.array_equal(s.table.pairs, table0.pairs)):
                raise ValueError("all systems of one engine must share the residue tables")
        # crowder species: one type per distinct crowder radius over all
        # systems (a system's own species numbering is mapped onto these)
        radii: List[float] = []
        for s in self.systems:
            for r in s.crowder_radii():
                if r not in radii:
                    radii.append(r)
        if len(radii) > MAX_TYPES - NUM_AMINO:
            raise ValueError("at most %d distinct crowder radii" % (MAX_TYPES - NUM_AMINO))
        self._species = {r: NUM_AMINO + i for i, r in enumerate(radii)}
        self._topo = []
        descs = (SystemDesc * len(self.systems))()
        for i, s in enumerate(self.systems):
            mol_start, roles, types = s.topology()
            local = s.crowder_radii()
            if local:
                remap = np.arange(MAX_TYPES, dtype=np.int32)
                for k, r in enumerate(local):
                    remap[NUM_AMINO + k] = self._species[r]
                types = remap[types]
            self._topo.append((mol_start, roles, types))
            d = descs[i]
            d.n_beads = s.n_beads
            d.n_mol = s.n_mol
            d.n_replicas = self.n_replicas[i]
            d.mol_start = _ptr(mol_start, C.c_int)
            d.mol_role = _ptr(roles, C.c_int)
            d.bead_type = _ptr(types, C.c_int)
            d.box = s.box
            d.translate_only_crowders = 1 if s.translate_only_crowders else 0
        h = C.c_void_p()
        check(lib().remc_create(descs, len(self.systems), C.byref(self.params), C.byref(h)))
        self._h = h
        self.n_inst = lib().remc_num_instances(h)
        self.inst_system = np.repeat(np.arange(len(self.systems)), self.n_replicas)
        self.inst_slot = np.concatenate([np.arange(r) for r in self.n_replicas])
        self.inst_first = np.concatenate([[0], np.cumsum(self.n_replicas)[:-1]]).astype(int)
        self.set_type_tables()
        self.upload_state()

    # ------------------------------------------------------------ lifecycle
    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().remc_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ set-up
    def type_tables(self):
        vdw, q, rho = self.systems[0].type_tables()
        for r, t in self._species.items():
            rho[t] = np.float32(r)
        return vdw, q, rho, np.ascontiguousarray(self.systems[0].table.pairs, np.float32)

    def set_type_tables(self) -> None:
        vdw, q, rho, pairs = self.type_tables()
        check(lib().remc_set_type_tables(self._h, _ptr(vdw, C.c_float), _ptr(q, C.c_float),
                                         _ptr(rho, C.c_float), _ptr(pairs, C.c_float)))

    def set_params(self, params: Params) -> None:
        self.params = params
        check(lib().remc_set_params(self._h, C.byref(params)))

    def upload_state(self, pos=None, rel=None, centre=None, quat=None) -> None:
        """Per-instance state (concatenated in instance order); defaults to
        every replica holding its system's coordinates."""
        if pos is None:
            parts = [[], [], [], []]
            for s, r in zip(self.systems, self.n_replicas):
                st = s.state()
                for k in range(4):
                    parts[k].extend([st[k]] * r)
            pos, rel, centre, quat = [np.concatenate(p) for p in parts]
        pos = np.ascontiguousarray(pos, np.float32)
        rel = np.ascontiguousarray(rel, np.float32)
        centre = np.ascontiguousarray(centre, np.float32)
        quat = np.ascontiguousarray(quat, np.float64)
        check(lib().remc_upload_state(self._h, _ptr(pos, C.c_float), _ptr(rel, C.c_float),
                                      _ptr(centre, C.c_float), _ptr(quat, C.c_double)))

    def set_replica_params(self, ladders, translate_steps, rotate_steps) -> None:
        """ladders: per system, an increasing array of R temperatures;
        translate/rotate steps: per instance (or per system, broadcast)."""
        lad = np.concatenate([np.asarray(l, np.float32) for l in ladders]).astype(np.float32)
        ts = np.asarray(translate_steps, np.float32)
        rs = np.asarray(rotate_steps, np.float64)
        if ts.size == len(self.systems):
            ts = np.repeat(ts, self.n_replicas)
        if rs.size == len(self.systems):
            rs = np.repeat(rs, self.n_replicas)
        ts = np.ascontiguousarray(ts, np.float32)
        rs = np.ascontiguousarray(rs, np.float64)
        if lad.size != self.n_inst or ts.size != self.n_inst or rs.size != self.n_inst:
            raise ValueError("replica parameter arrays must have one entry per instance")
        check(lib().remc_set_replica_params(self._h, _ptr(lad, C.c_float), _ptr(ts, C.c_float),
                                            _ptr(rs, C.c_double)))
        self.ladder = lad

    # ------------------------------------------------------------ compute
    def energy_full(self) -> np.ndarray:
        out = np.zeros(self.n_inst, np.float64)
        check(lib().remc_energy_full(self._h, _ptr(out, C.c_double)))
        return out

    def energies(self) -> np.ndarray:
        out = np.zeros(self.n_inst, np.float64)
        check(lib().remc_get_energies(self._h, _ptr(out, C.c_double)))
        return out

    def sweep(self, n_steps: int, seed: int, step0: int = 0) -> None:
        check(lib().remc_sweep(self._h, n_steps, seed, step0))

    def sweep_plain(self, n_steps: int, seed: int, step0: int = 0) -> None:
        check(lib().remc_sweep_plain(self._h, n_steps, seed, step0))

    def exchange(self, seed: int, round_: int, offset: int) -> None:
        check(lib().remc_exchange(self._h, seed, round_, offset))

    def run(self, n_blocks: int, steps_per_block: int, seed: int, step0: int = 0,
            round0: int = 0) -> None:
        check(lib().remc_run(self._h, n_blocks, steps_per_block, seed, step0, round0))

    def sync(self) -> None:
        check(lib().remc_sync(self._h))

    def delta_energy(self, inst: int, mol: int, new_pos: np.ndarray) -> float:
        p = np.ascontiguousarray(new_pos, np.float32).reshape(-1)
        out = C.c_double(0.0)
        check(lib().remc_delta_energy(self._h, inst, mol, _ptr(p, C.c_float), C.byref(out)))
        return out.value

    # ------------------------------------------------------------ read back
    def download_state(self, out=None):
        """(pos, rel, centre, quat) of every instance; `out` = four C-contiguous
        arrays of those shapes and types to fill instead (e.g. pinned memory)."""
        nb = sum(s.n_beads * r for s, r in zip(self.systems, self.n_replicas))
        nm = sum(s.n_mol * r for s, r in zip(self.systems, self.n_replicas))
        if out is not None:
            pos, rel, cen, quat = out
            for a, shape, dt in ((pos, (nb, 3), np.float32), (rel, (nb, 3), np.float32),
                                 (cen, (nm, 3), np.float32), (quat, (nm, 4), np.float64)):
                if a.shape != shape or a.dtype != dt or not a.flags.c_contiguous:
                    raise ValueError("download_state: out arrays must be %s %s" % (shape, dt))
        else:
            pos = np.zeros((nb, 3), np.float32)
            rel = np.zeros((nb, 3), np.float32)
            cen = np.zeros((nm, 3), np.float32)
            quat = np.zeros((nm, 4), np.float64)
        check(lib().remc_download_state(self._h, _ptr(pos, C.c_float), _ptr(rel, C.c_float),
                                        _ptr(cen, C.c_float), _ptr(quat, C.c_double)))
        return pos, rel, cen, quat

    def instance_slices(self):
        """(bead slice, molecule slice) of every instance in the flat arrays."""
        out = []
        b = m = 0
        for s, r in zip(self.systems, self.n_replicas):
            for _ in range(r):
                out.append((slice(b, b + s.n_beads), slice(m, m + s.n_mol)))
                b += s.n_beads
                m += s.n_mol
        return out

    def temperature_map(self) -> np.ndarray:
        out = np.zeros(self.n_inst, np.int32)
        check(lib().remc_get_temperature_map(self._h, _ptr(out, C.c_int)))
        return out

    def set_temperature_map(self, temp_of_slot) -> None:
        t = np.ascontiguousarray(temp_of_slot, np.int32)
        check(lib().remc_set_temperature_map(self._h, _ptr(t, C.c_int)))

    def set_energies(self, energy, noncrowder=None) -> None:
        """Restore the running energies (checkpoint resume)."""
        e = np.ascontiguousarray(energy, np.float64)
        c = None if noncrowder is None else np.ascontiguousarray(noncrowder, np.float64)
        check(lib().remc_set_energies(self._h, _ptr(e, C.c_double),
                                      None if c is None else _ptr(c, C.c_double)))

    def counters(self):
        a = np.zeros(self.n_inst, np.int32)
        b = np.zeros(self.n_inst, np.int32)
        r = np.zeros(self.n_inst, np.int32)
        check(lib().remc_get_counters(self._h, _ptr(a, C.c_int), _ptr(b, C.c_int),
                                      _ptr(r, C.c_int)))
        return a, b, r

    def reset_counters(self) -> None:
        check(lib().remc_reset_counters(self._h))

    # ------------------------------------------------------------ sampling
    def set_sampling(self, sample_every: int, sample_after: int = 0,
                     bound_threshold: float = -1.1844, max_records: int = 0,
                     max_poses: int = 0) -> None:
        """Replica::sample inside the sweeps; see remc_set_sampling."""
        self._max_records, self._max_poses = max_records, max_poses
        check(lib().remc_set_sampling(self._h, sample_every, sample_after, bound_threshold,
                                      max_records, max_poses))

    def sample_counters(self):
        n = np.zeros(self.n_inst, np.int32)
        b = np.zeros(self.n_inst, np.int32)
        check(lib().remc_get_sample_counters(self._h, _ptr(n, C.c_int), _ptr(b, C.c_int)))
        return n, b

    def read_samples(self):
        """(records, poses, dropped): records as dicts, poses as (n, 7) array
        of quaternion w,x,y,z and centre x,y,z."""
        mr = max(1, getattr(self, "_max_records", 0))
        mp = max(1, getattr(self, "_max_poses", 0))
        recs = (SampleRecord * mr)()
        poses = (SamplePose * mp)()
        nr, npz, nd = C.c_int(0), C.c_int(0), C.c_int(0)
        check(lib().remc_read_samples(self._h, recs, mr, poses, mp, C.byref(nr), C.byref(npz),
                                      C.byref(nd)))
        out = [{"inst": r.inst, "label": r.label, "e_noncrowder": r.e_noncrowder,
                "e_total": r.e_total, "temperature": r.temperature, "n_mol": r.n_mol,
                "pose_offset": r.pose_offset} for r in recs[:nr.value]]
        arr = np.array([list(p.q) + list(p.centre) for p in poses[:npz.value]], np.float64)
        return out, arr.reshape(-1, 7), nd.value

    def adjoint(self):
        """Forces, per-molecule force/torque, dE/dlambda, dE/dXi, dE/deps[20x20]
        and the energy of every instance (remc_energy_adjoint)."""
        nb = sum(s.n_beads * r for s, r in zip(self.systems, self.n_replicas))
        nm = sum(s.n_mol * r for s, r in zip(self.systems, self.n_replicas))
        f = np.zeros((nb, 3), np.float32)
        ft = np.zeros((nm, 6), np.float64)
        dl = np.zeros(self.n_inst)
        dx = np.zeros(self.n_inst)
        de = np.zeros((self.n_inst, 20, 20))
        e = np.zeros(self.n_inst)
        check(lib().remc_energy_adjoint(self._h, _ptr(f, C.c_float), _ptr(ft, C.c_double),
                                        _ptr(dl, C.c_double), _ptr(dx, C.c_double),
                                        _ptr(de, C.c_double), _ptr(e, C.c_double)))
        return {"forces": f, "mol_force_torque": ft, "dE_dlambda": dl, "dE_dxi": dx,
                "dE_deps": de, "energy": e}

    def dE_dlambda(self) -> np.ndarray:
        """dE/dlambda of every instance only (no forces copied back)."""
        dl = np.zeros(self.n_inst)
        check(lib().remc_energy_adjoint(self._h, None, None, _ptr(dl, C.c_double), None, None,
                                        None))
        return dl

    def energy_full_async(self) -> None:
        """Enqueue the full energy without reading it back."""
        check(lib().remc_energy_full(self._h, None))

    def adjoint_kernels(self) -> None:
        """Run the adjoint without copying its outputs back."""
        check(lib().remc_energy_adjoint(self._h, None, None, None, None, None, None))

    def noncrowder_energies(self) -> np.ndarray:
        out = np.zeros(self.n_inst, np.float64)
        check(lib().remc_get_noncrowder_energies(self._h, _ptr(out, C.c_double)))
        return out

    def pair_evaluations(self):
        """(residue-residue, crowder) pair evaluations since the last reset."""
        a = C.c_uint64(0)
        b = C.c_uint64(0)
        check(lib().remc_get_pair_evaluations(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def autotune(self, probe_steps: int = 200, seed: int = 12345):
        """Pick the fastest sweep schedule for these systems (remc_autotune);
        returns (threads, molecule data in shared memory, probe ms)."""
        t, m, ms = C.c_int(0), C.c_int(0), C.c_float(0.0)
        check(lib().remc_autotune(self._h, probe_steps, seed, C.byref(t), C.byref(m),
                                  C.byref(ms)))
        return t.value, bool(m.value), ms.value

    def set_cluster(self, cluster: int) -> None:
        """CTAs per replica (a thread-block cluster of 1, 2, 4 or 8)."""
        check(lib().remc_set_cluster(self._h, cluster))

    def schedule(self):
        """(threads per replica, centres in shared memory, CTAs per replica)."""
        t, m, c = C.c_int(), C.c_int(), C.c_int()
        check(lib().remc_get_schedule(self._h, C.byref(t), C.byref(m), C.byref(c)))
        return t.value, bool(m.value), c.value

    def set_work_order(self, by_cost: bool) -> None:
        """Persistent sweep work order: by each block's proposal costs (True,
        the default) or the static order (False); results are identical."""
        check(lib().remc_set_work_order(self._h, 1 if by_cost else 0))

    def work_order(self):
        """(by cost, kernel launches per sweep launch)."""
        b, n = C.c_int(), C.c_int()
        check(lib().remc_get_work_order(self._h, C.byref(b), C.byref(n)))
        return bool(b.value), n.value

    def set_schedule(self, threads: int, mol_in_smem: bool) -> None:
        check(lib().remc_set_schedule(self._h, threads, 1 if mol_in_smem else 0))

    def set_bead_storage(self, shared: bool) -> None:
        """Beads resident in shared memory (True) or updated in place in
        global memory (False; any system size, same results)."""
        check(lib().remc_set_bead_storage(self._h, 1 if shared else 0))

    def fold_flags(self) -> np.ndarray:
        """Per system: 1 when the sweep folds the minimum image (see
        remc_get_fold_flags)."""
        out = np.zeros(len(self.systems), np.int32)
        check(lib().remc_get_fold_flags(self._h, _ptr(out, C.c_int)))
        return out

    def beads_in_shared_memory(self) -> bool:
        v = C.c_int()
        check(lib().remc_get_bead_storage(self._h, C.byref(v)))
        return bool(v.value)

    def stream_ptr(self) -> int:
        """The handle's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        s = C.c_void_p(0)
        check(lib().remc_get_stream(self._h, C.byref(s)))
        return int(s.value or 0)
