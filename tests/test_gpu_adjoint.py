"""GPU adjoint of the MLS-MPM substep (CrB200SolverAdjointRecord / AdjointBackward) through the
torch.autograd.Function wrapper.

The reference has no gradient path.  The GPU gradients (float32) are compared with the FP64 host
adjoint (oracle/adjoint_fp64.py), which the CPU tests pin to central finite differences within
1e-5: dL/dE, dL/dnu and the summed dL/dv0 within 1e-3 relative, per-particle dL/dv0 within 1e-2
relative L2, with the kinematic contact model and with the effective-mass model (two-body impulses
against a dynamic shape).  Central finite differences of the GPU forward itself, all in deterministic mode
(CRB200_OPT_DETERMINISTIC, which the backward pass's replays follow), are checked within 1e-3 for
E, nu and v0 on the small cube, and for E and nu over the 200 substeps of the
material-identification workload (64k particles), whose gradients are also checked against the
FP64 host adjoint.
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


@pytest.mark.parametrize("kind", ["plane", "mixed", "effmass"])
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


def _fd_median(f, step):
    """Median of the central differences (f(s) - f(-s)) / 2s at s = step, step / 2, step / 4.

    The forward map is piecewise smooth with small jumps: a grid node's contact switches on where
    its advected position crosses a shape surface while approaching it (the normal velocity is
    removed at once), and a node whose mass crosses the 1e-4 cutoff switches between keeping its
    momentum and dividing by its mass.  The adjoint holds those branch decisions fixed, as a
    derivative must; a difference whose interval holds a jump is off by the jump over 2s.  The median
    of three steps drops one such difference."""
    ds = [(f(s) - f(-s)) / (2 * s) for s in (step, step / 2, step / 4)]
    return float(np.median(ds)), ds


def _central_difference_check(sc, steps, caps, K, E_at=E0, nu_at=NU0, h=1e-2, dv_step=2e-3, tol=1e-3,
                              tol_nu=None, check_v0=True):
    """GPU adjoint gradients dL/dE, dL/dnu and the summed dL/dv0 against central differences of
    the GPU forward itself, everything in CRB200_OPT_DETERMINISTIC: the recorded forward, the
    replays of the backward pass and the perturbed forwards all sum in a fixed order, so the
    differences carry no run-to-run scatter and the gradient belongs to the very function that is
    differenced.  What is left in a difference is the float32 rounding of the forward (a jitter
    that grows as 1/h), truncation (h^2) and the forward's jumps (`_fd_median`): the steps are
    1 %, 0.5 % and 0.25 % of E and nu and 2, 1 and 0.5 mm/s for v0.  Targets come from another
    material (E 3e4, nu 0.3) so that the loss depends strongly on E and nu; the loss is summed in
    float64."""
    import torch

    n = sc.n
    cb.build_library()
    ds = cb.DeviceScene(sc, compute_initial=False)
    ds.solver.set_option(cb.OPT_DETERMINISTIC, 1)
    ds.compute_initial_data()
    dev = ds.device
    run = Trajectory(ds, steps, caps, checkpoint_interval=K)

    def fwd(E, nu, dv=0.0):
        lam, mu = lame(torch.tensor(E, dtype=torch.float64, device=dev), torch.tensor(nu, dtype=torch.float64, device=dev))
        v0 = torch.tensor(sc.vel[:, :3] + dv, dtype=torch.float32, device=dev)
        return run.forward(lam.float().expand(n), mu.float().expand(n), v0)

    T = fwd(3e4, 0.3).double()
    # deterministic: the same forward twice is the same bit for bit
    assert torch.equal(fwd(E_at, nu_at), fwd(E_at, nu_at))

    def L(E=E_at, nu=nu_at, dv=0.0):
        return float(((fwd(E, nu, dv).double() - T) ** 2).mean(dim=(1, 2)).sum())

    Et = torch.tensor(E_at, dtype=torch.float64, device=dev, requires_grad=True)
    nut = torch.tensor(nu_at, dtype=torch.float64, device=dev, requires_grad=True)
    v0 = torch.tensor(sc.vel[:, :3], dtype=torch.float32, device=dev, requires_grad=True)
    lam, mu = lame(Et, nut)
    pos = trajectory(run, lam.float().expand(n), mu.float().expand(n), v0)
    ((pos.double() - T) ** 2).mean(dim=(1, 2)).sum().backward()
    gE, gnu, gv = float(Et.grad), float(nut.grad), v0.grad.double().sum(0).cpu().numpy()
    fE, dsE = _fd_median(lambda t: L(E=E_at * (1 + t)), h)
    fnu, dsnu = _fd_median(lambda t: L(nu=nu_at * (1 + t)), h)
    fE, fnu = fE / E_at, fnu / nu_at
    tol_nu = tol if tol_nu is None else tol_nu
    print(f"ADJOINT n={n} steps={steps} dE rel={abs(gE - fE) / abs(fE):.3e} (differences {[d / E_at for d in dsE]}) "
          f"dnu rel={abs(gnu - fnu) / abs(fnu):.3e} (differences {[d / nu_at for d in dsnu]}) gE={gE:.6e} gnu={gnu:.6e}")
    assert abs(gE - fE) <= tol * abs(fE), (gE, fE)
    assert abs(gnu - fnu) <= tol_nu * abs(fnu), (gnu, fnu)
    if not check_v0:
        return
    for k in range(3):
        e = np.zeros(3)
        e[k] = 1.0
        fv, dsv = _fd_median(lambda t: L(dv=e * t), dv_step)
        print(f"ADJOINT dv0[{k}] gpu={gv[k]:.6e} fd={fv:.6e} (differences {dsv})")
        assert abs(gv[k] - fv) <= tol * max(abs(fv), 0.1 * np.abs(gv).max()), (k, gv[k], fv)


def test_gpu_adjoint_matches_central_differences():
    """120 substeps of impact of the small adjoint cube: gradients within 1e-3 of central
    differences."""
    _central_difference_check(scenes.adjoint_scene("plane"), 120, (40, 80, 120), 20)


def _material_id_scene():
    """The material-identification workload: the 64k-particle cube (0.4 m, dx 0.02, 8 ppc) 1 cm
    above the ground at -1 m/s, substeps of 2e-4 s, at the initial guess E 8e3, nu 0.25."""
    return scenes.material_cube(E=8e3, nu=0.25, drop=0.01, v0=(0.0, -1.0, 0.0))


def test_gpu_adjoint_material_identification_central_differences():
    """The whole 200 substeps of the material-identification workload (captures at 50, 100, 150,
    200, checkpoints every 20): dL/dE within 1e-3 and dL/dnu within 2e-3 of central differences
    of the GPU forward.  Over 150 substeps of contact of 64k particles the forward's jumps are
    dense: the differences for nu scatter by about 1e-3 from one step size to the next, and for
    v0 (which moves the impact itself) every step size holds many jumps, so the v0 gradient of
    this workload is checked against the FP64 adjoint instead (next test)."""
    _central_difference_check(_material_id_scene(), 200, (50, 100, 150, 200), 20, E_at=8e3, nu_at=0.25,
                              tol_nu=2e-3, check_v0=False)


def test_gpu_adjoint_material_identification_against_fp64():
    """The material-identification workload against the FP64 host adjoint, targets made at E 2e4,
    nu 0.35.  The FP64 host adjoint of all 64k particles runs at about 3 s per substep, so the
    check covers the first 100 substeps (captures at 50 and 100, the impact included): dL/dE and
    dL/dnu within 1e-3, the summed dL/dv0 within 5e-3 and per-particle dL/dv0 within 1e-2
    relative L2.  The float32 and FP64 trajectories part by about 2e-5 of the displacement, enough
    to switch some nodes' contact branches (see `_fd_median`), and with them a part of the v0
    gradient: measured 3.3e-3 on the summed dL/dv0."""
    import torch

    sc = _material_id_scene()
    steps, caps, K = 100, (50, 100), 20
    n = sc.n
    cb.build_library()
    ds = cb.DeviceScene(sc)
    dev = ds.device
    run = Trajectory(ds, steps, caps, checkpoint_interval=K)
    lt, mt = lame(2e4, 0.35)
    tgt_gpu = run.forward(torch.full((n,), lt, device=dev), torch.full((n,), mt, device=dev),
                          torch.tensor(sc.vel[:, :3], device=dev)).double()
    tgt = {t: tgt_gpu[k].cpu().numpy() for k, t in enumerate(caps)}
    # FP64 host adjoint at the guess
    a = Fp64Adjoint(sc)
    lam0, mu0 = lame(8e3, 0.25)
    xs = a.forward(np.full(n, lam0), np.full(n, mu0), sc.vel[:, :3], steps)
    g = a.backward({t: 2.0 * (xs[t - 1] - tgt[t]) / (3 * n) for t in caps})
    (dlE, dlnu), (dmE, dmnu) = lame_grad(8e3, 0.25)
    fE = float((g["g_lam"] * dlE + g["g_mu"] * dmE).sum())
    fnu = float((g["g_lam"] * dlnu + g["g_mu"] * dmnu).sum())
    fv = g["g_v0"]
    # GPU adjoint through the autograd wrapper
    Et = torch.tensor(8e3, dtype=torch.float64, device=dev, requires_grad=True)
    nut = torch.tensor(0.25, dtype=torch.float64, device=dev, requires_grad=True)
    v0 = torch.tensor(sc.vel[:, :3], dtype=torch.float32, device=dev, requires_grad=True)
    lam, mu = lame(Et, nut)
    pos = trajectory(run, lam.float().expand(n), mu.float().expand(n), v0)
    T = torch.tensor(np.stack([tgt[t] for t in caps]), dtype=torch.float32, device=dev)
    position_mse(pos, T).backward()
    gE, gnu, gv = float(Et.grad), float(nut.grad), v0.grad.double().cpu().numpy()
    scale = max(float(np.abs(xs[-1] - sc.pos_mass[:, :3]).max()), sc.cell_size)
    sv, fsv = gv.sum(0), fv.sum(0)
    print(f"ADJOINT cfg5 n={n} steps={steps} forward {np.abs(pos[-1].detach().cpu().numpy() - xs[-1]).max() / scale:.3e} "
          f"dE rel={abs(gE - fE) / abs(fE):.3e} dnu rel={abs(gnu - fnu) / abs(fnu):.3e} "
          f"dv0 sum rel={np.abs(sv - fsv).max() / np.abs(fsv).max():.3e} "
          f"dv0 L2 rel={np.linalg.norm(gv - fv) / np.linalg.norm(fv):.3e}")
    assert abs(gE - fE) <= 1e-3 * abs(fE), (gE, fE)
    assert abs(gnu - fnu) <= 1e-3 * abs(fnu), (gnu, fnu)
    assert float(np.abs(sv - fsv).max()) <= 5e-3 * float(np.abs(fsv).max()), (sv, fsv)
    assert np.linalg.norm(gv - fv) <= 1e-2 * np.linalg.norm(fv)


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
