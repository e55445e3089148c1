"""GPU tests of the reference-ABI drop-ins (include/remc_reference_abi.h),
through ctypes with device buffers in the reference's own layout."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden_system

pytestmark = pytest.mark.gpu

E_RTOL = 1e-5


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _energy(system, block=32):
    import torch
    from remcdockingsimulator_b200.reference_abi import abi, pack_reference_layout
    L = abi()
    pos, meta = pack_reference_layout(system, block)
    dp, dm = _dev(pos), _dev(meta)
    table = np.ascontiguousarray(system.table.pairs, np.float32)
    dt = torch.zeros(400, dtype=torch.float32, device="cuda")
    L.copyLJPotentialDataToDevice(C.c_void_p(dt.data_ptr()), table.ctypes.data)
    assert L.remc_reference_abi_status() == 0
    L.CUDA_setBoxDimension(system.box)
    out = C.c_double(0.0)
    L.CUDA_EonDevice(C.c_void_p(dp.data_ptr()), C.c_void_p(dm.data_ptr()), None, None, None,
                     C.c_void_p(dt.data_ptr()), C.byref(out), block, pos.shape[0], 0)
    assert L.remc_reference_abi_status() == 0
    return out.value, (dp, dm, dt, pos)


def test_eondevice_golden_structures(golden, golden_table, built_lib):
    for k, st in enumerate(golden["structures"]):
        s = golden_system(golden, golden_table, k)
        e, _ = _energy(s, 64)
        ref = st["reference_E"]
        if abs(ref) > 1e-2:
            assert abs(e - ref) / abs(ref) < E_RTOL, (k, e, ref)
        else:
            assert abs(e - ref) < 1e-6


def test_eondevice_crowded_vs_reference_engine(built_lib):
    """Crowders in the reference model ((6/r)^6 inside 15 A) against the
    reference's own Replica::E()."""
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    w = synth.crowded(4)
    s = w.systems[0]
    e, _ = _energy(s, 32)
    if ob.reference_available():
        ref = ob.ReferenceReplica(s).E()
    else:
        from remcdockingsimulator_b200.engine import make_params
        ref = ob.FP64Oracle(s, make_params()).energy(s.state()[0])
    assert abs(e - ref) <= E_RTOL * max(abs(ref), 1e-3), (e, ref)


def test_eondevice_async_grid_sums_to_energy(built_lib):
    import torch
    from remcdockingsimulator_b200.reference_abi import abi
    from remcdockingsimulator_b200 import synth, model
    w = synth.two_chain(8)
    s = w.systems[0]
    e_sync, (dp, dm, dt, pos) = _energy(s, 32)
    L = abi()
    grid = (pos.shape[0] // 32)
    res = torch.full((grid * grid,), 7.0, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    L.CUDA_EonDevice_async(C.c_void_p(dp.data_ptr()), C.c_void_p(dm.data_ptr()), None, None, None,
                           C.c_void_p(dt.data_ptr()), C.c_void_p(res.data_ptr()), grid, 32,
                           pos.shape[0], 0, C.c_void_p(stream.cuda_stream))
    stream.synchronize()
    assert L.remc_reference_abi_status() == 0
    # Replica::SumGridResults: float sum of the grid times KBTConversionFactor
    host = res.cpu().numpy()
    total = np.float32(0.0)
    for v in host:
        total = np.float32(total + v)
    e_async = float(np.float32(total * model.KBT_CONVERSION_FACTOR))
    assert abs(e_async - e_sync) <= 1e-5 * max(abs(e_sync), 1e-3)


def test_bound_table_and_errors(built_lib):
    from remcdockingsimulator_b200.reference_abi import abi
    from remcdockingsimulator_b200 import synth
    L = abi()
    s = synth.two_chain(2).systems[0]
    e_explicit, (dp, dm, dt, pos) = _energy(s, 32)
    L.bindLJTexture(C.c_void_p(dt.data_ptr()))
    out = C.c_double(0.0)
    L.CUDA_EonDevice(C.c_void_p(dp.data_ptr()), C.c_void_p(dm.data_ptr()), None, None, None, None,
                     C.byref(out), 32, pos.shape[0], 0)
    assert L.remc_reference_abi_status() == 0
    assert out.value == e_explicit
    L.unbindLJTexture()
    L.CUDA_EonDevice(C.c_void_p(dp.data_ptr()), C.c_void_p(dm.data_ptr()), None, None, None, None,
                     C.byref(out), 32, pos.shape[0], 0)
    assert L.remc_reference_abi_status() != 0
    L.CUDA_setBoxDimension(-1.0)
    assert L.remc_reference_abi_status() != 0


def test_translate_and_rotate_molecule(built_lib):
    import torch
    from remcdockingsimulator_b200.reference_abi import abi, pack_reference_layout
    from remcdockingsimulator_b200 import synth
    L = abi()
    s = synth.two_chain(6).systems[0]
    pos, meta = pack_reference_layout(s, 32)
    m = s.molecules[1]
    start = s.molecules[0].n
    dp = _dev(pos)
    d_start = torch.tensor([start], dtype=torch.int32, device="cuda")
    d_len = torch.tensor([m.n], dtype=torch.int32, device="cuda")
    centre = np.array([*m.centre, 0.0], np.float32)
    d_c = _dev(centre)
    t = np.array([1.5, -2.0, 0.25, 0.0], np.float32)
    d_t = _dev(t)
    L.CUDA_translateMolecule(C.c_void_p(dp.data_ptr()), C.c_void_p(d_start.data_ptr()),
                             C.c_void_p(d_len.data_ptr()), m.n, C.c_void_p(d_t.data_ptr()),
                             C.c_void_p(d_c.data_ptr()), None)
    torch.cuda.synchronize()
    got = dp.cpu().numpy()
    assert np.allclose(got[start:start + m.n, :3], pos[start:start + m.n, :3] + t[:3], atol=1e-5)
    assert np.allclose(got[:start], pos[:start])
    assert np.allclose(d_c.cpu().numpy()[:3], centre[:3] + t[:3], atol=1e-5)
    # rotation by pi about z through the (moved) centre flips x and y offsets
    rv = _dev(np.array([0.0, 0.0, 1.0, np.pi], np.float32))
    c_now = d_c.cpu().numpy()
    before = dp.cpu().numpy()[start:start + m.n, :3]
    L.CUDA_rotateMolecule(C.c_void_p(dp.data_ptr()), C.c_void_p(d_start.data_ptr()),
                          C.c_void_p(d_len.data_ptr()), m.n, C.c_void_p(rv.data_ptr()),
                          C.c_void_p(d_c.data_ptr()), None)
    torch.cuda.synchronize()
    after = dp.cpu().numpy()[start:start + m.n, :3]
    off = before - c_now[:3]
    exp = np.stack([-off[:, 0], -off[:, 1], off[:, 2]], axis=1) + c_now[:3]
    assert np.allclose(after, exp, atol=1e-3)


def test_eondevice_concurrent_streams_and_threads(built_lib):
    """Energies of two different systems queued at the same time from two host
    threads, on two streams (CUDA_EonDevice_async) and on the default stream
    (CUDA_EonDevice), equal the energies of the same calls made one at a
    time: every stream has its own partial sums, and synchronous calls take
    turns on theirs."""
    import threading
    import torch
    from conftest import crowder_lattice
    from remcdockingsimulator_b200.reference_abi import abi, pack_reference_layout
    L = abi()
    systems = [crowder_lattice(16000, seed=11, side=26), crowder_lattice(12000, seed=12, side=26)]
    assert systems[0].box == systems[1].box  # the box is one process-wide setting
    L.CUDA_setBoxDimension(systems[0].box)
    dev = []
    for s in systems:
        pos, meta = pack_reference_layout(s, 32)
        table = np.ascontiguousarray(s.table.pairs, np.float32).reshape(-1)
        dev.append((_dev(pos), _dev(meta), _dev(table), pos.shape[0]))

    def sync_energy(k):
        dp, dm, dt, n = dev[k]
        out = C.c_double(0.0)
        L.CUDA_EonDevice(C.c_void_p(dp.data_ptr()), C.c_void_p(dm.data_ptr()), None, None, None,
                         C.c_void_p(dt.data_ptr()), C.byref(out), 32, n, 0)
        assert L.remc_reference_abi_status() == 0
        return out.value

    def async_energy(k, stream, res):
        dp, dm, dt, n = dev[k]
        L.CUDA_EonDevice_async(C.c_void_p(dp.data_ptr()), C.c_void_p(dm.data_ptr()), None, None,
                               None, C.c_void_p(dt.data_ptr()), C.c_void_p(res.data_ptr()), 1, 32,
                               n, 0, C.c_void_p(stream.cuda_stream))
        assert L.remc_reference_abi_status() == 0

    alone_sync = [sync_energy(0), sync_energy(1)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    alone_async = []
    for k in range(2):
        r = torch.zeros(1, dtype=torch.float32, device="cuda")
        async_energy(k, streams[k], r)
        streams[k].synchronize()
        alone_async.append(float(r.item()))
    assert alone_async[0] != alone_async[1]

    reps = 24
    got_async = [[torch.zeros(1, dtype=torch.float32, device="cuda") for _ in range(reps)]
                 for _ in range(2)]
    got_sync = [[None] * reps for _ in range(2)]
    errors = []

    def worker(k):
        try:
            torch.cuda.set_device(0)
            for i in range(reps):
                async_energy(k, streams[k], got_async[k][i])
                got_sync[k][i] = sync_energy(k)
        except Exception as exc:  # reported below
            errors.append(exc)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    torch.cuda.synchronize()
    assert not errors, errors
    for k in range(2):
        assert all(v == alone_sync[k] for v in got_sync[k]), (k, got_sync[k], alone_sync[k])
        vals = [float(r.item()) for r in got_async[k]]
        assert all(v == alone_async[k] for v in vals), (k, vals, alone_async[k])
