"""GPU test of CUDA_EonDevice_noalloc, the allocation-free energy entry point.

Some callers cannot call cudaMalloc: a host whose GPU memory is reserved by
another allocator, or a Monte Carlo loop that cannot pay for cudaMalloc /
cudaFree's implicit device synchronisation on every step. For them the
library offers one entry point that keeps its partial sums in a fixed device
array instead of allocating. This test drives it through the C ABI (ctypes)
with caller-owned device buffers and checks, on two calls in a row, that it
returns what the allocating CUDA_EonDevice returns (within the 1e-5 relative
tolerance of the other energy tests), and that sizes beyond its fixed limit
are refused with an error.

The file is named so that pytest collects it after every other test file.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_RTOL = 1e-5


def _upload(system, block=32):
    import torch
    from remcdockingsimulator_b200.reference_abi import abi, pack_reference_layout
    L = abi()
    pos, meta = pack_reference_layout(system, block)
    dp = torch.from_numpy(pos).cuda()
    dm = torch.from_numpy(meta).cuda()
    dt = torch.from_numpy(np.ascontiguousarray(system.table.pairs, np.float32).reshape(-1)).cuda()
    return L, pos, dp, dm, dt


def _allocating_energy(L, system, pos, dp, dm, dt, block=32):
    L.CUDA_setBoxDimension(system.box)
    out = C.c_double(0.0)
    L.CUDA_EonDevice(C.c_void_p(dp.data_ptr()), C.c_void_p(dm.data_ptr()), None, None, None,
                     C.c_void_p(dt.data_ptr()), C.byref(out), block, pos.shape[0], 0)
    assert L.remc_reference_abi_status() == 0
    return out.value


def test_noalloc_matches_allocating_entry_point(built_lib):
    import torch
    from remcdockingsimulator_b200 import synth
    systems = [synth.crowded(31).systems[0], synth.two_chain(32).systems[0]]
    result = torch.zeros(1, dtype=torch.float64, device="cuda")
    for s in systems:  # two calls in a row, reusing the shared scratch
        L, pos, dp, dm, dt = _upload(s)
        expected = _allocating_energy(L, s, pos, dp, dm, dt)
        stream = torch.cuda.current_stream()
        rc = L.CUDA_EonDevice_noalloc(C.c_void_p(dp.data_ptr()), C.c_void_p(dm.data_ptr()),
                                      C.c_void_p(dt.data_ptr()), pos.shape[0],
                                      C.c_void_p(result.data_ptr()),
                                      C.c_void_p(stream.cuda_stream))
        assert rc == 0, L.remc_last_error_string()
        torch.cuda.synchronize()
        got = float(result.item())
        assert abs(got - expected) <= E_RTOL * max(abs(expected), 1e-3), (got, expected)


def test_noalloc_rejects_sizes_beyond_its_limit(built_lib):
    import torch
    from remcdockingsimulator_b200.reference_abi import abi
    L = abi()
    too_many = 32641  # REMC_NOALLOC_MAX_BEADS + 1
    dp = torch.zeros((too_many, 4), dtype=torch.float32, device="cuda")
    dm = torch.zeros((too_many, 4), dtype=torch.float32, device="cuda")
    dt = torch.zeros(400, dtype=torch.float32, device="cuda")
    result = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = L.CUDA_EonDevice_noalloc(C.c_void_p(dp.data_ptr()), C.c_void_p(dm.data_ptr()),
                                  C.c_void_p(dt.data_ptr()), too_many,
                                  C.c_void_p(result.data_ptr()), None)
    assert rc != 0
    assert b"exceeds" in L.remc_last_error_string()
