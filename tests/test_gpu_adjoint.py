"""GPU adjoint of the MLS-MPM substep (CrB200SolverAdjointRecord / AdjointBackward) through the
torch.autograd.Function wrapper.

The reference has no gradient path.  The GPU gradients (float32) are compared with the FP64 host
adjoint (oracle/adjoint_fp64.py), which the CPU tests pin to central finite differences within
1e-5: dL/dE, dL/dnu and the summed dL/dv0 within 1e-3 relative, per-particle dL/dv0 within 1e-2
relative L2.  Central finite differences of the GPU forward itself are checked within 1e-3 (E) and
2e-3 (nu, v0).
"""
import numpy as np
import pytest

from conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

import crmpm_b200 as cb  # noqa: E402
from adjoint_fp64 import Fp64Adjoint, lame_grad  # noqa: E402
from crmpm_b200 import scenes  # noqa: E402
from crmpm_b200.adjoint import Trajectory, lame, position_mse, trajectory  # noqa: E402

STEPS = 30
CAPS = (10, 20, 30)
E0, NU0 = 2e4, 0.35


def _targets(sc, seed=7):
    """FP64 trajectory of the scene at (E0, NU0) plus noise: the identification targets."""
    n = sc.n
    a = Fp64Adjoint(sc)
    lam, mu = lame(E0, NU0)
    xs = a.forward(np.full(n, lam), np.full(n, mu), sc.vel[:, :3], STEPS)
    rng = np.random.default_rng(seed)
    return a, xs, {t: xs[t - 1] + rng.normal(0.0, 1e-3, xs[t - 1].shape) for t in CAPS}


def _fp64_grads(a, xs, tgt, n):
    g = a.backward({t: 2.0 * (xs[t - 1] - tgt[t]) / (3 * n) for t in CAPS})
    (dlE, dlnu), (dmE, dmnu) = lame_grad(E0, NU0)
    return (float((g["g_lam"] * dlE + g["g_mu"] * dmE).sum()), float((g["g_lam"] * dlnu + g["g_mu"] * dmnu).sum()),
            g["g_v0"])


def _gpu_loss_and_grads(ds, run, sc, tgt, E=E0, nu=NU0, dv=None):
    import torch

    n = sc.n
    dev = ds.device
    Et = torch.tensor(E, dtype=torch.float64, device=dev, requires_grad=True)
    nut = torch.tensor(nu, dtype=torch.float64, device=dev, requires_grad=True)
    v0 = torch.tensor(sc.vel[:, :3] + (0 if dv is None else dv), dtype=torch.float32, device=dev, requires_grad=True)
    lam, mu = lame(Et, nut)
    pos = trajectory(run, lam.float().expand(n), mu.float().expand(n), v0)
    T = torch.tensor(np.stack([tgt[t] for t in CAPS]), dtype=torch.float32, device=dev)
    loss = position_mse(pos, T)
    loss.backward()
    return (float(loss.detach()), float(Et.grad), float(nut.grad), v0.grad.double().cpu().numpy(),
            pos.detach().cpu().numpy())


def _run(sc):
    cb.build_library()
    ds = cb.DeviceScene(sc)
    return ds, Trajectory(ds, STEPS, CAPS, checkpoint_interval=8)


@pytest.mark.parametrize("kind", ["plane", "mixed"])
def test_gpu_adjoint_matches_fp64_adjoint(kind):
    sc = scenes.adjoint_scene(kind)
    a, xs, tgt = _targets(sc)
    gE, gnu, gv = _fp64_grads(a, xs, tgt, sc.n)
    ds, run = _run(sc)
    _, E_g, nu_g, v_g, pos = _gpu_loss_and_grads(ds, run, sc, tgt)
    # forward: float32 engine vs FP64 host, relative to the displacement scale
    scale = max(float(np.abs(xs[-1] - sc.pos_mass[:, :3]).max()), sc.cell_size)
    assert float(np.abs(pos[-1] - xs[-1]).max()) / scale < 1e-4
    assert abs(E_g - gE) <= 1e-3 * abs(gE), (E_g, gE)
    assert abs(nu_g - gnu) <= 1e-3 * abs(gnu), (nu_g, gnu)
    np.testing.assert_allclose(v_g.sum(0), gv.sum(0), rtol=1e-3, atol=1e-3 * np.abs(gv.sum(0)).max())
    assert np.linalg.norm(v_g - gv) <= 1e-2 * np.linalg.norm(gv)


def test_gpu_adjoint_matches_central_differences():
    """Central differences of the GPU forward itself, on 120 substeps of impact with targets made at
    another material (E 3e4, nu 0.3) so that the loss depends strongly on E and nu.  Steps: 0.3 %
    of E and nu, 1e-3 m/s for v0; the loss is summed in float64.  The float32 forward sums with
    atomics in a varying order, so one central difference scatters by up to 1.2e-3 between runs
    while the adjoint itself repeats to 1e-5: the E and nu differences are averaged over two
    evaluations and held to 2e-3, v0 to 2e-3."""
    import torch

    steps, caps = 120, (40, 80, 120)
    sc = scenes.adjoint_scene("plane")
    n = sc.n
    cb.build_library()
    ds = cb.DeviceScene(sc)
    dev = ds.device
    run = Trajectory(ds, steps, caps, checkpoint_interval=20)

    def fwd(E, nu, dv=0.0):
        lam, mu = lame(torch.tensor(E, dtype=torch.float64, device=dev), torch.tensor(nu, dtype=torch.float64, device=dev))
        v0 = torch.tensor(sc.vel[:, :3] + dv, dtype=torch.float32, device=dev)
        return run.forward(lam.float().expand(n), mu.float().expand(n), v0)

    T = fwd(3e4, 0.3).double()

    def L(E=E0, nu=NU0, dv=0.0):
        return float(((fwd(E, nu, dv).double() - T) ** 2).mean(dim=(1, 2)).sum())

    Et = torch.tensor(E0, dtype=torch.float64, device=dev, requires_grad=True)
    nut = torch.tensor(NU0, dtype=torch.float64, device=dev, requires_grad=True)
    v0 = torch.tensor(sc.vel[:, :3], dtype=torch.float32, device=dev, requires_grad=True)
    lam, mu = lame(Et, nut)
    pos = trajectory(run, lam.float().expand(n), mu.float().expand(n), v0)
    ((pos.double() - T) ** 2).mean(dim=(1, 2)).sum().backward()
    gE, gnu, gv = float(Et.grad), float(nut.grad), v0.grad.double().sum(0).cpu().numpy()
    h = 3e-3
    fE = sum((L(E=E0 * (1 + h)) - L(E=E0 * (1 - h))) / (2 * E0 * h) for _ in range(2)) / 2
    fnu = sum((L(nu=NU0 * (1 + h)) - L(nu=NU0 * (1 - h))) / (2 * NU0 * h) for _ in range(2)) / 2
    assert abs(gE - fE) <= 2e-3 * abs(fE), (gE, fE)
    assert abs(gnu - fnu) <= 2e-3 * abs(fnu), (gnu, fnu)
    for k in range(3):
        dv = np.zeros(3)
        dv[k] = 1e-3
        fv = (L(dv=dv) - L(dv=-dv)) / 2e-3
        assert abs(gv[k] - fv) <= 2e-3 * max(abs(fv), 0.1 * np.abs(gv).max()), (k, gv[k], fv)


def test_gpu_adjoint_leaves_final_state_and_repeats():
    """Backward leaves the recorded final state; a second record + backward gives the same gradients."""
    sc = scenes.adjoint_scene("plane")
    _, _, tgt = _targets(sc)
    ds, run = _run(sc)
    r1 = _gpu_loss_and_grads(ds, run, sc, tgt)
    st = ds.state()
    np.testing.assert_allclose(st["x"], r1[4][-1], atol=0)
    r2 = _gpu_loss_and_grads(ds, run, sc, tgt)
    assert abs(r1[1] - r2[1]) <= 1e-4 * abs(r1[1])
    np.testing.assert_allclose(r1[3], r2[3], rtol=1e-3, atol=1e-4 * np.abs(r1[3]).max())


def test_batched_adjoint_matches_scenes_alone():
    import torch

    sl = [scenes.adjoint_scene("plane", seed=1006), scenes.adjoint_scene("mixed", seed=1007)]
    b = cb.DeviceBatch(sl)
    run = Trajectory(b, STEPS, CAPS, checkpoint_interval=8)
    n = b.scene.n
    dev = b.device
    rng = np.random.default_rng(3)
    g = torch.tensor(rng.normal(0, 1.0, (len(CAPS), n, 3)), dtype=torch.float32, device=dev)
    lam = torch.tensor(b.scene.mat_params[:, 0], device=dev)
    mu = torch.tensor(b.scene.mat_params[:, 1], device=dev)
    v0 = torch.tensor(b.scene.vel[:, :3], device=dev)
    run.forward(lam, mu, v0)
    gl, gm, gv = (t.cpu().numpy() for t in run.backward(g))
    for s, sc in enumerate(sl):
        sl_ = b.batch.slice(s)
        ds = cb.DeviceScene(sc)
        r1 = Trajectory(ds, STEPS, CAPS, checkpoint_interval=8)
        r1.forward(lam[sl_], mu[sl_], v0[sl_])
        gl1, gm1, gv1 = (t.cpu().numpy() for t in r1.backward(g[:, sl_].contiguous()))
        for got, ref in ((gl[sl_], gl1), (gm[sl_], gm1), (gv[sl_], gv1)):
            assert np.linalg.norm(got - ref) <= 1e-3 * np.linalg.norm(ref) + 1e-12


def test_adjoint_refuses_what_it_does_not_differentiate():
    sc = scenes.cube_drop(solver=scenes.SOLVER_PB, dt=0.002)
    ds = cb.DeviceScene(sc)
    with pytest.raises(cb.CrmpmError, match="MLS"):
        Trajectory(ds, 4, (4,)).forward(*[__import__("torch").zeros(sc.n, device=ds.device)] * 2,
                                        __import__("torch").zeros((sc.n, 3), device=ds.device))
    sc = scenes.contact_scene("trimesh")
    ds = cb.DeviceScene(sc)
    import torch

    with pytest.raises(cb.CrmpmError, match="shapes"):
        Trajectory(ds, 4, (4,)).forward(torch.tensor(sc.mat_params[:, 0], device=ds.device),
                                        torch.tensor(sc.mat_params[:, 1], device=ds.device),
                                        torch.zeros((sc.n, 3), device=ds.device))
