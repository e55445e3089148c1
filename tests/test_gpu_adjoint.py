"""GPU adjoint (remc_energy_adjoint) against the FP64 oracle's analytic adjoint,
which tests/test_adjoint_cpu.py pins to FP64 central finite differences; and a
torch.autograd.Function over the engine's energy, used only here as the
gradient harness."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(name, seed, mode_ref=False, w=None):
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import Engine, make_params
    w = synth.WORKLOADS[name](seed) if w is None else w
    s = w.systems[0]
    p = make_params(lambda_=0.16) if mode_ref else w.params
    R = 2
    with Engine([s], R, p) as eng:
        eng.set_replica_params([w.ladders[0][:R]], np.full(R, 0.5, np.float32), np.full(R, 0.2))
        eng.energy_full()
        eng.sweep(300, seed, 0)  # move away from the generated layout
        st = eng.download_state()
        full = eng.energy_full()
        adj = eng.adjoint()
        sl = eng.instance_slices()
    o = ob.FP64Oracle(s, p)
    for k in range(R):
        bs, ms = sl[k]
        pos = st[0][bs]
        f, dl, dx, de = o.adjoint(pos)
        fg = adj["forces"][bs].astype(np.float64)
        err = np.linalg.norm(fg - f) / max(np.linalg.norm(f), 1e-12)
        assert err < 2e-4, (k, err)
        big = np.abs(f) > 1e-2 * np.abs(f).max()
        assert np.allclose(fg[big], f[big], rtol=2e-3, atol=1e-6)
        assert abs(adj["dE_dlambda"][k] - dl) <= 1e-4 * max(abs(dl), 1e-6), (adj["dE_dlambda"][k], dl)
        assert abs(adj["dE_dxi"][k] - dx) <= 1e-4 * max(abs(dx), 1e-8), (adj["dE_dxi"][k], dx)
        deg = adj["dE_deps"][k]
        assert np.allclose(deg, de[:20, :20], rtol=1e-4, atol=1e-5 * np.abs(de).max())
        assert abs(adj["energy"][k] - full[k]) <= 1e-5 * max(abs(full[k]), 1e-3)
        # per-molecule force and torque about the centre from the oracle forces
        ms_ = s.topology()[0]
        rel = st[1][bs].astype(np.float64)
        ft = adj["mol_force_torque"][ms]
        for m in range(s.n_mol):
            a, b = ms_[m], ms_[m + 1]
            F = f[a:b].sum(axis=0)
            tq = np.cross(rel[a:b], f[a:b]).sum(axis=0)
            scale = max(np.abs(f[a:b]).max(), 1e-9)
            assert np.allclose(ft[m, :3], F, atol=2e-3 * scale * (b - a) ** 0.5 + 1e-6)
            assert np.allclose(ft[m, 3:], tq, atol=2e-3 * scale * 30 * (b - a) ** 0.5 + 1e-5)


def test_adjoint_crowded_r12(built_lib):
    _check("crowded", 21)


def test_adjoint_crowded_reference_crowders(built_lib):
    """The reference's crowder model: (6/r)^6 walls cut at 15 A."""
    _check("crowded", 23, mode_ref=True)


def test_adjoint_two_chain(built_lib):
    _check("two_chain", 22)


def test_torch_autograd_harness(built_lib):
    """E(pos) through the engine as a torch.autograd.Function; its gradient is
    the adjoint's -F and matches FP64 central differences of the oracle."""
    import torch
    from oracle import bindings as ob
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import Engine

    w = synth.two_chain(23)
    s = w.systems[0]
    eng = Engine([s], 1, w.params)
    eng.set_replica_params([w.ladders[0][:1]], [0.5], [0.2])
    _, rel, cen, quat = s.state()

    class RemcEnergy(torch.autograd.Function):
        @staticmethod
        def forward(ctx, pos):
            p32 = pos.detach().cpu().numpy().astype(np.float32)
            eng.upload_state(p32, rel, cen, quat)
            adj = eng.adjoint()
            ctx.save_for_backward(torch.from_numpy(-adj["forces"].astype(np.float64)))
            return torch.tensor(float(adj["energy"][0]), dtype=torch.float64)

        @staticmethod
        def backward(ctx, g):
            (grad,) = ctx.saved_tensors
            return g * grad

    pos = torch.from_numpy(s.state()[0].astype(np.float64)).requires_grad_(True)
    E = RemcEnergy.apply(pos)
    E.backward()
    o = ob.FP64Oracle(s, w.params)
    p0 = s.state()[0]
    fd = []
    grads = pos.grad.numpy()
    for b in np.argsort(-np.abs(grads).max(axis=1))[:5]:
        for c in range(3):
            pp, pm = p0.copy(), p0.copy()
            pp[b, c] = np.float32(p0[b, c] + 1e-3)
            pm[b, c] = np.float32(p0[b, c] - 1e-3)
            d = (o.energy(pp) - o.energy(pm)) / (float(pp[b, c]) - float(pm[b, c]))
            assert abs(d - grads[b, c]) <= 3e-3 * max(abs(d), 1e-2), (b, c, d, grads[b, c])
    eng.close()
