"""ctypes binding of the engine's C ABI (include/remc_b200.h).

The shared library is built in-tree (remcdockingsimulator_b200/lib/) by
`python -m remcdockingsimulator_b200.build`. Loading fails loudly when it is
missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

from .build import LIB

REMC_OK = 0
REMC_ERR_INVALID = -1
REMC_ERR_CUDA = -2
REMC_ERR_NOMEM = -3
REMC_ERR_STATE = -4
REMC_ERR_NUMERIC = -5
REMC_ERR_TIMEOUT = -6
MAX_TYPES = 24
NUM_AMINO = 20


class RemcError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__("remc error %d: %s" % (code, message))
        self.code = code


class Params(C.Structure):
    _fields_ = [("lambda_", C.c_float), ("e0", C.c_float), ("debye_length", C.c_float),
                ("dh_const", C.c_float), ("lj_cf", C.c_float), ("kbt_cf", C.c_float),
                ("crowder_mode", C.c_int), ("crowder_cutoff", C.c_float),
                ("crowder_eps", C.c_float)]


class SampleRecord(C.Structure):
    _fields_ = [("inst", C.c_int), ("label", C.c_uint32), ("e_noncrowder", C.c_double),
                ("e_total", C.c_double), ("temperature", C.c_float), ("n_mol", C.c_int),
                ("pose_offset", C.c_int)]


class SamplePose(C.Structure):
    _fields_ = [("q", C.c_double * 4), ("centre", C.c_float * 3)]


class SystemDesc(C.Structure):
    _fields_ = [("n_beads", C.c_int), ("n_mol", C.c_int), ("n_replicas", C.c_int),
                ("mol_start", C.POINTER(C.c_int)), ("mol_role", C.POINTER(C.c_int)),
                ("bead_type", C.POINTER(C.c_int)), ("box", C.c_float),
                ("translate_only_crowders", C.c_int)]


_lib = None

P = C.c_void_p
PF = C.POINTER(C.c_float)
PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int)

_SIGS = {
    "remc_default_params": (None, [C.POINTER(Params)]),
    "remc_create": (C.c_int, [C.POINTER(SystemDesc), C.c_int, C.POINTER(Params), C.POINTER(P)]),
    "remc_destroy": (C.c_int, [P]),
    "remc_set_params": (C.c_int, [P, C.POINTER(Params)]),
    "remc_set_type_tables": (C.c_int, [P, PF, PF, PF, PF]),
    "remc_upload_state": (C.c_int, [P, PF, PF, PF, PD]),
    "remc_download_state": (C.c_int, [P, PF, PF, PF, PD]),
    "remc_set_replica_params": (C.c_int, [P, PF, PF, PD]),
    "remc_energy_full": (C.c_int, [P, PD]),
    "remc_get_energies": (C.c_int, [P, PD]),
    "remc_sweep": (C.c_int, [P, C.c_int, C.c_uint64, C.c_uint32]),
    "remc_sweep_plain": (C.c_int, [P, C.c_int, C.c_uint64, C.c_uint32]),
    "remc_exchange": (C.c_int, [P, C.c_uint64, C.c_uint32, C.c_int]),
    "remc_get_temperature_map": (C.c_int, [P, PI]),
    "remc_set_temperature_map": (C.c_int, [P, PI]),
    "remc_set_energies": (C.c_int, [P, PD, PD]),
    "remc_get_counters": (C.c_int, [P, PI, PI, PI]),
    "remc_reset_counters": (C.c_int, [P]),
    "remc_delta_energy": (C.c_int, [P, C.c_int, C.c_int, PF, PD]),
    "remc_run": (C.c_int, [P, C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_uint32]),
    "remc_sync": (C.c_int, [P]),
    "remc_get_pair_evaluations": (C.c_int, [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "remc_get_stream": (C.c_int, [P, C.POINTER(C.c_void_p)]),
    "remc_set_sampling": (C.c_int, [P, C.c_int, C.c_uint32, C.c_double, C.c_int, C.c_int]),
    "remc_get_sample_counters": (C.c_int, [P, PI, PI]),
    "remc_read_samples": (C.c_int, [P, C.POINTER(SampleRecord), C.c_int, C.POINTER(SamplePose),
                                    C.c_int, PI, PI, PI]),
    "remc_get_noncrowder_energies": (C.c_int, [P, PD]),
    "remc_energy_adjoint": (C.c_int, [P, PF, PD, PD, PD, PD, PD]),
    "remc_num_instances": (C.c_int, [P]),
    "remc_autotune": (C.c_int, [P, C.c_int, C.c_uint64, PI, PI, PF]),
    "remc_set_schedule": (C.c_int, [P, C.c_int, C.c_int]),
    "remc_set_cluster": (C.c_int, [P, C.c_int]),
    "remc_get_schedule": (C.c_int, [P, PI, PI, PI]),
    "remc_set_work_order": (C.c_int, [P, C.c_int]),
    "remc_get_work_order": (C.c_int, [P, PI, PI]),
    "remc_set_bead_storage": (C.c_int, [P, C.c_int]),
    "remc_get_bead_storage": (C.c_int, [P, PI]),
    "remc_check_wait_timeout": (C.c_int, [P, C.c_int]),
    "remc_get_fold_flags": (C.c_int, [P, PI]),
    "remc_last_error_string": (C.c_char_p, []),
    "remc_post_rebuild": (C.c_int, [PF, PI, C.c_int, PI, PF, C.c_float, PD, PF, C.c_int, PF, PF]),
    "remc_post_drms": (C.c_int, [PF, C.c_int, PF, PI, C.c_int, C.c_int, C.c_float, C.c_float, PD,
                                 C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                 C.POINTER(C.c_longlong)]),
}


def lib() -> C.CDLL:
    """Load libremc_b200.so (once). Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(
                "libremc_b200.so not found at %s: build it with "
                "`python -m remcdockingsimulator_b200.build` (no CPU fallback exists)" % LIB)
        L = C.CDLL(LIB)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != REMC_OK:
        msg = lib().remc_last_error_string()
        raise RemcError(code, msg.decode() if msg else "")


def default_params() -> Params:
    p = Params()
    lib().remc_default_params(C.byref(p))
    return p
