"""ctypes binding of include/remc_reference_abi.h (the reference's CUDA C ABI
drop-ins) and a packer for the reference's device layout.

`pack_reference_layout` builds the two float4 arrays Replica::ReplicaDataToDevice
fills (simulation engine/src/Replica.cpp:1308-1417): positions with the molecule
index in w and padding beads (w = -2) up to a multiple of the block size, and
metadata (residue type, charge, vdW radius, molecule role). Crowder beads
carry type -1 (Molecule::setMoleculeRoleIdentifier, Molecule.cpp:120-142).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import lib as _lib

P = C.c_void_p
_bound = False


def abi() -> C.CDLL:
    global _bound
    L = _lib()
    if not _bound:
        sig = {
            "LJPotentialDataToDevice": (C.c_void_p, [C.c_void_p]),
            "copyLJPotentialDataToDevice": (None, [P, P]),
            "CUDA_EonDevice": (None, [P, P, P, P, P, P, C.POINTER(C.c_double), C.c_int, C.c_int,
                                      C.c_int]),
            "CUDA_EonDevice_async": (None, [P, P, P, P, P, P, P, C.c_int, C.c_int, C.c_int,
                                            C.c_int, P]),
            "CUDA_rotateMolecule": (None, [P, P, P, C.c_int, P, P, P]),
            "CUDA_translateMolecule": (None, [P, P, P, C.c_int, P, P, P]),
            "CUDA_setBoxDimension": (None, [C.c_float]),
            "CUDA_freeBoxDimension": (None, []),
            "bindLJTexture": (None, [P]),
            "unbindLJTexture": (None, []),
            "remc_reference_abi_status": (C.c_int, []),
            "CUDA_EonDevice_noalloc": (C.c_int, [P, P, P, C.c_int, P, P]),
            "CUDA_memcpy_to_device": (C.c_int, [P, P, C.c_int]),
            "CUDA_memcpy_to_host": (C.c_int, [P, P, C.c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _bound = True
    return L


def pack_reference_layout(system, block_size: int = 32):
    """(positions, metadata) float32 arrays [P, 4], P = bead count rounded up
    to a multiple of block_size."""
    n = system.n_beads
    Pn = int(np.ceil(n / block_size) * block_size)
    pos = np.zeros((Pn, 4), np.float32)
    meta = np.zeros((Pn, 4), np.float32)
    pos[:, 3] = -2.0
    meta[:, 0] = 20.0  # PADDER_AATYPE
    b = 0
    for m, mol in enumerate(system.molecules):
        for k in range(mol.n):
            pos[b, :3] = mol.pos[k]
            pos[b, 3] = float(m)
            t = int(mol.types[k]) if not mol.crowder else 0
            meta[b, 0] = -1.0 if mol.crowder else float(t)
            meta[b, 1] = system.table.charge[t]
            meta[b, 2] = system.table.vdw[t]
            meta[b, 3] = -1.0 if mol.crowder else 0.0
            b += 1
    return pos, meta
