"""GPU test of CUDA_EonDevice_noalloc, the allocation-free energy entry point.

Some callers cannot call cudaMalloc: a host whose GPU memory is reserved by
another allocator, or a Monte Carlo loop that cannot pay for cudaMalloc /
cudaFree's implicit device synchronisation on every step. For them the
library offers one entry point that keeps its partial sums in a fixed device
array instead of allocating. This test drives it through the C ABI (ctypes)
with caller-owned device buffers and checks, on two calls in a row, that it
returns what the allocating CUDA_EonDevice returns and what the FP64 oracle
computes (within the 1e-5 relative tolerance of the other energy tests);
that the largest size it accepts (REMC_NOALLOC_MAX_BEADS beads, whose last
tile pair writes the array's last used slot) is right; that it uses the table
bound by bindLJTexture when given none; and that sizes beyond its fixed limit
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


def _noalloc(L, dp, dm, dt, n, result, table=True):
    import torch
    stream = torch.cuda.current_stream()
    rc = L.CUDA_EonDevice_noalloc(C.c_void_p(dp.data_ptr()), C.c_void_p(dm.data_ptr()),
                                  C.c_void_p(dt.data_ptr()) if table else None, n,
                                  C.c_void_p(result.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert rc == 0, L.remc_last_error_string()
    torch.cuda.synchronize()
    return float(result.item())


def _oracle_energy(system):
    from oracle import bindings as ob
    from remcdockingsimulator_b200.engine import make_params
    # the reference layout's model: the reference's constants, (6/r)^6 crowders
    return ob.FP64Oracle(system, make_params()).energy(system.state()[0])


def _close(got, ref):
    return abs(got - ref) <= E_RTOL * max(abs(ref), 1e-3)


def test_noalloc_matches_allocating_entry_point_and_oracle(built_lib):
    import torch
    from remcdockingsimulator_b200 import synth
    systems = [synth.crowded(31).systems[0], synth.two_chain(32).systems[0]]
    result = torch.zeros(1, dtype=torch.float64, device="cuda")
    for s in systems:  # two calls in a row, reusing the shared scratch
        L, pos, dp, dm, dt = _upload(s)
        expected = _allocating_energy(L, s, pos, dp, dm, dt)
        got = _noalloc(L, dp, dm, dt, pos.shape[0], result)
        assert _close(got, expected), (got, expected)
        ref = _oracle_energy(s)
        assert _close(got, ref), (got, ref)


def test_noalloc_at_its_largest_size(built_lib):
    """REMC_NOALLOC_MAX_BEADS = 32640 beads: 255 tiles of 128, 32640 tile
    pairs, the last of them in the array's last used slot."""
    import torch
    from conftest import crowder_lattice
    s = crowder_lattice(32640)
    L, pos, dp, dm, dt = _upload(s)
    assert pos.shape[0] == 32640
    L.CUDA_setBoxDimension(s.box)
    result = torch.zeros(1, dtype=torch.float64, device="cuda")
    got = _noalloc(L, dp, dm, dt, pos.shape[0], result)
    ref = _oracle_energy(s)
    assert ref > 1.0
    assert _close(got, ref), (got, ref)
    expected = _allocating_energy(L, s, pos, dp, dm, dt)
    assert _close(got, expected), (got, expected)


def test_noalloc_uses_the_bound_table(built_lib):
    import torch
    from remcdockingsimulator_b200 import synth
    s = synth.two_chain(33).systems[0]
    L, pos, dp, dm, dt = _upload(s)
    L.CUDA_setBoxDimension(s.box)
    result = torch.zeros(1, dtype=torch.float64, device="cuda")
    explicit = _noalloc(L, dp, dm, dt, pos.shape[0], result)
    L.bindLJTexture(C.c_void_p(dt.data_ptr()))
    try:
        bound = _noalloc(L, dp, dm, dt, pos.shape[0], result, table=False)
    finally:
        L.unbindLJTexture()
    assert bound == explicit
    assert _close(bound, _oracle_energy(s))


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
