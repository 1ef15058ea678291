"""Parity at the workloads' own horizons.

The other parity tests keep the runs short.  These run the headline scenes for the number of
substeps (or steps) the workloads are defined over, and every test prints and asserts the bar it
applies, next to the reference's own deviation that the bar is derived from:

* the 1.6M-particle MLS tissue slab, 500 substeps, against the reference's own CUDA solver, with
  the bar set by the reference's own sensitivity to the order of its float sums (the same
  reference run on the particles listed in another order);
* a reduced slab (0.3 x 0.1 x 0.3 m, dx 0.01, pins and probe kept), 500 substeps, against the FP64
  oracle and the reference's float32 arithmetic (`e_ref` = the reference float32 run's own
  departure from FP64);
* PB-MPM cutting (a slab cut by a quad-slicer blade off the grid planes), 300 steps, against FP64
  and the reference's CUDA solver, with the slicer cut masks checked bit for bit on identical float
  inputs at sampled steps;
* a 64-scene MLS batch, 200 substeps, against the same scenes run alone.

Position metric: max_p |x - x_ref| / max(max_p |x_ref - x0|, dx).
"""
import dataclasses
import threading

import numpy as np
import pytest

from conftest import cuda_available
from gpu_helpers import rel_pos_err

import oracle_py as op  # noqa: E402

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

import crmpm_b200 as cb  # noqa: E402
from crmpm_b200 import scenes  # noqa: E402


def _report(name, **vals):
    """One line per test with the errors measured and the bar applied (shown with pytest -rA)."""
    print(f"PARITY {name} " + " ".join(f"{k}={v:.3e}" if isinstance(v, float) else f"{k}={v}"
                                       for k, v in vals.items()))


def _engine(sc, steps):
    cb.build_library()
    g = cb.DeviceScene(sc)
    g.step(steps)
    st = g.state()
    st["force"], st["torque"] = g.coupling()
    return st


def _threaded(*fns):
    """Runs the oracle loops side by side (their C calls release the GIL)."""
    out = [None] * len(fns)

    def run(k):
        out[k] = fns[k]()

    ts = [threading.Thread(target=run, args=(k,)) for k in range(len(fns))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    return out


def _quantiles(x, x_ref, x0, dx):
    """Per-particle position error over max(displacement, dx): median, 99th, 99.9th percentile, max."""
    scale = max(float(np.abs(x_ref - x0).max()), dx)
    err = np.abs(x - x_ref).max(axis=1) / scale
    return [float(q) for q in np.quantile(err, (0.5, 0.99, 0.999, 1.0))]


def _permuted(sc, seed=11):
    """The same scene with its particles listed in a seeded random order (and the inverse order)."""
    perm = np.random.default_rng(seed).permutation(sc.n)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(sc.n)
    return dataclasses.replace(sc, pos_mass=sc.pos_mass[perm], vel=sc.vel[perm], mat_params=sc.mat_params[perm],
                               mat_type=sc.mat_type[perm], mask=sc.mask[perm]), inv


@pytest.mark.skipif(not op.ref_gpu_available(), reason="oracle/_ref/ref_gpu_driver not built")
def test_full_slab_500_substeps_against_reference_cuda(tmp_path):
    """Over 500 substeps the pinned slab amplifies float32 rounding: a change in the order of the
    node sums moves particles near the pins by up to about 1e-2 of the displacement scale (the
    reference's float32 arithmetic and the FP64 oracle part that far on the reduced slab below).
    Two runs of the reference's CUDA solver mostly repeat its atomic order, so they are no measure
    of that.  The measure is the reference run on the same particles listed in another order (its
    atomics then sum in another order).  The engine differs from the reference's CUDA build by more
    than an order of sums: it sums each cell's particles in registers before any atomic, and rounds
    the stencil arithmetic as the reference's CPU build does instead of with the CUDA build's
    contracted multiply-adds.  So its distance to the reference must stay within three times the
    order spread, quantile by quantile (median, 99th, 99.9th percentile, max), or within 1e-4; the
    reduced slab below checks that the engine and the reference's float32 arithmetic are equally
    far from FP64."""
    sc = scenes.tissue_slab()
    steps = 500
    ref = op.ref_gpu_run(sc, steps, workdir=str(tmp_path))
    psc, inv = _permuted(sc)
    rp = op.ref_gpu_run(psc, steps, workdir=str(tmp_path))
    ref_p = {"x": rp["x"][inv], "v": rp["v"][inv]}
    got = _engine(sc, steps)
    x0 = sc.pos_mass[:, :3]
    q_ord = np.array(_quantiles(ref_p["x"], ref["x"], x0, sc.cell_size))
    q_got = np.array(_quantiles(got["x"], ref["x"], x0, sc.cell_size))
    tol = np.maximum(1e-4, 3.0 * q_ord)
    vscale = max(float(np.abs(ref["v"]).max()), 1e-3)
    dv_ord = float(np.abs(ref_p["v"] - ref["v"]).max())
    dv = float(np.abs(got["v"] - ref["v"]).max())
    vtol = max(1e-3 * vscale, 2.0 * dv_ord)
    _report("slab1.6M_500_vs_refcuda", e_median=q_got[0], e_p99=q_got[1], e_p999=q_got[2], e_max=q_got[3],
            order_median=q_ord[0], order_p99=q_ord[1], order_p999=q_ord[2], order_max=q_ord[3],
            tol_max=float(tol[3]), dv=dv, dv_order=dv_ord, vtol=vtol, disp=float(np.abs(ref["x"] - x0).max()))
    for name, e, t in zip(("median", "p99", "p99.9", "max"), q_got, tol):
        assert e <= t, f"engine vs reference CUDA, {name}: {e:.3e} > {t:.3e}"
    assert dv <= vtol
    S = sc.shapes.shape_type.shape[0]
    for key in ("force", "torque"):
        a, b = got[key][:S], ref[key][:S]
        scale = max(float(np.abs(b).max()), 1e-6)
        assert float(np.abs(a - b).max()) <= 1e-3 * scale, key


def _reduced_slab():
    return scenes.tissue_slab(size=(0.3, 0.1, 0.3), cell=0.01, bounds_min=(-0.2, -0.05, -0.2),
                              bounds_max=(0.2, 0.25, 0.2))


def test_reduced_slab_500_substeps_against_fp64():
    sc = _reduced_slab()
    steps = 500
    got = _engine(sc, steps)

    def fp64():
        o = op.PortOracle(sc, 64)
        o.compute_initial_data()
        o.step(steps)
        return o.state()

    def ref32():
        r = op.RefOracle(sc) if op.ref_available() else op.PortOracle(sc, 32)
        r.compute_initial_data()
        r.step(steps)
        return r.state()

    b, c = _threaded(fp64, ref32)
    x0 = sc.pos_mass[:, :3]
    e_ref = rel_pos_err(c["x"], b["x"], x0, sc.cell_size)
    tol = max(1e-4, 2.0 * e_ref)
    e64 = rel_pos_err(got["x"], b["x"], x0, sc.cell_size)
    e32 = rel_pos_err(got["x"], c["x"], x0, sc.cell_size)
    df_ref = float(np.abs(c["F"] - b["F"]).max())
    df = float(np.abs(got["F"] - b["F"]).max())
    ftol = max(1e-4, 2.0 * df_ref)
    q64 = _quantiles(got["x"], b["x"], x0, sc.cell_size)
    qref = _quantiles(c["x"], b["x"], x0, sc.cell_size)
    _report("slab_reduced_500_vs_fp64", n=sc.n, e64=e64, e32=e32, e_ref=e_ref, tol=tol, dF=df, dF_ref=df_ref,
            ftol=ftol, e64_median=q64[0], e64_p99=q64[1], ref_median=qref[0], ref_p99=qref[1])
    assert e64 <= tol, f"engine vs FP64 {e64:.3e} > {tol:.3e} (reference float32 vs FP64: {e_ref:.3e})"
    assert e32 <= tol, f"engine vs reference float32 {e32:.3e} > {tol:.3e}"
    assert df <= ftol


OFF_GRID = np.array([0.29, 0.37, 0.41], np.float32)  # blade offset from the grid planes, in cells


@pytest.mark.skipif(not op.ref_gpu_available(), reason="oracle/_ref/ref_gpu_driver not built")
def test_pb_cutting_300_steps(tmp_path):
    """A PB-MPM slab (0.12 x 0.04 x 0.12 m, dx 0.008, 10 solver iterations) cut by a quad-slicer
    blade inside it, 300 steps: cut masks bit for bit against the oracle on the engine's own
    positions every 50 steps, and positions after 300 steps against FP64 and the reference's CUDA
    solver within max(2e-3, 2 x the reference CUDA run's own departure from FP64)."""
    sc = scenes.pb_cutting(size=(0.12, 0.04, 0.12), cell=0.008, bounds_min=(-0.12, -0.1, -0.12),
                           bounds_max=(0.12, 0.1, 0.12), iterations=10)
    sc.shapes.position[1, :3] = np.array([0.0, -0.01, 0.0], np.float32) + OFF_GRID * np.float32(sc.cell_size)
    steps, every = 300, 50
    cb.build_library()
    g = cb.DeviceScene(sc)
    checker = op.PortOracle(sc, 32)
    cut_particles = 0
    for k in range(steps // every):
        # the masks a step uses are those of the positions it starts from
        g.step(every - 1)
        g.sync()
        x = g.pos[: sc.n, :3].cpu().numpy()
        g.step(1, graph=False)
        masks = g.cut_masks()
        checker.set_state(x=x.astype(np.float64))
        np.testing.assert_array_equal(masks, checker.cut_masks(), err_msg=f"cut masks of step {(k + 1) * every}")
        cut_particles = max(cut_particles, int(np.count_nonzero(masks)))
    assert cut_particles > 0, "the blade cuts no particle"
    got = g.state()

    def fp64():
        o = op.PortOracle(sc, 64)
        o.compute_initial_data()
        o.step(steps)
        return o.state()

    x64 = fp64()["x"]
    ref = op.ref_gpu_run(sc, steps, workdir=str(tmp_path))
    x0 = sc.pos_mass[:, :3]
    e_ref = rel_pos_err(ref["x"], x64, x0, sc.cell_size)
    tol = max(2e-3, 2.0 * e_ref)
    e64 = rel_pos_err(got["x"], x64, x0, sc.cell_size)
    eref = rel_pos_err(got["x"], ref["x"], x0, sc.cell_size)
    _report("pb_cut_300_steps", n=sc.n, e64=e64, e_refcuda=eref, e_ref=e_ref, tol=tol, cut=cut_particles)
    assert e64 <= tol, f"engine vs FP64 {e64:.3e} > {tol:.3e} (reference CUDA vs FP64: {e_ref:.3e})"
    assert eref <= tol


def test_batch_64_scenes_200_substeps_against_scenes_alone():
    """64 of the batch workload's scenes (2k-16k particles each) stepped together for 200
    substeps, each against the same scene alone on the single-scene solver."""
    cb.build_library()
    sl = scenes.batched_scenes(num_scenes=64, nmin=2000, nmax=16000)
    steps = 200
    b = cb.DeviceBatch(sl)
    b.step(steps)
    full = b.state()
    worst = (0.0, -1)
    worst_v = 0.0
    for s, sc in enumerate(sl):
        got = b.scene_state(s, full)
        g = cb.DeviceScene(sc)
        g.step(steps)
        ref = g.state()
        del g
        e = rel_pos_err(got["x"], ref["x"], sc.pos_mass[:, :3], sc.cell_size)
        vscale = max(float(np.abs(ref["v"]).max()), 1e-3)
        worst = max(worst, (e, s))
        worst_v = max(worst_v, float(np.abs(got["v"] - ref["v"]).max()) / vscale)
    _report("batch64_200_vs_alone", worst=worst[0], scene=worst[1], tol=1e-4, worst_v_rel=worst_v, vtol=1e-3)
    assert worst[0] <= 1e-4, f"scene {worst[1]}: position deviation {worst[0]:.3e}"
    assert worst_v <= 1e-3
