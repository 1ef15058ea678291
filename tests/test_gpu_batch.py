"""Batched scenes (CrB200BatchCreate): one solver advancing many independent scenes must give each
scene the result it gets when run alone, and the oracle's.

Scene-by-scene equality is not bitwise: grid nodes sum contributions from several CTAs with float
atomics, whose order varies from run to run.  Positions must agree within 1e-4 of
max(displacement, dx) (the single-scene parity tolerance) and slicer cut masks bit for bit.
"""
import numpy as np
import pytest

from conftest import cuda_available
from gpu_helpers import rel_pos_err

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

import crmpm_b200 as cb  # noqa: E402
import oracle_py as op  # noqa: E402
from crmpm_b200 import scenes  # noqa: E402

POS_TOL = 1e-4


def _alone(sc, steps):
    g = cb.DeviceScene(sc)
    g.step(steps)
    return g.state()


def _check_against_alone(scene_list, steps, graph=True, tol_scale=1.0):
    """Each scene of the batch vs the same scene alone: positions within tol_scale x 1e-4 of
    max(displacement, dx), velocities within tol_scale x 1e-3 of the velocity scale, F within
    tol_scale x 1e-4."""
    cb.build_library()
    b = cb.DeviceBatch(scene_list)
    b.step(steps, graph=graph)
    full = b.state()
    for s, sc in enumerate(scene_list):
        got = b.scene_state(s, full)
        ref = _alone(sc, steps)
        x0 = sc.pos_mass[:, :3]
        e = rel_pos_err(got["x"], ref["x"], x0, sc.cell_size)
        assert e <= tol_scale * POS_TOL, f"scene {s} ({sc.name}): position deviation {e:.3e}"
        vscale = max(float(np.abs(ref["v"]).max()), 1e-3)
        assert float(np.abs(got["v"] - ref["v"]).max()) <= tol_scale * 1e-3 * vscale + 1e-6, sc.name
        assert float(np.abs(got["F"] - ref["F"]).max()) <= tol_scale * 1e-4, sc.name
        np.testing.assert_allclose(got["V0"], ref["V0"], rtol=1e-6)
    return b


def test_mls_batch_matches_scenes_alone():
    """Heterogeneous bodies (plane + sphere each), 64^3-cell grids of 0.02 m."""
    _check_against_alone(scenes.batched_scenes(num_scenes=6, nmin=1500, nmax=8000), 60)


def test_mls_batch_matches_oracle():
    sl = scenes.batched_scenes(num_scenes=3, nmin=1500, nmax=4000)
    b = cb.DeviceBatch(sl)
    b.step(40)
    full = b.state()
    for s in (0, 2):
        o = op.PortOracle(sl[s], 64)
        o.compute_initial_data()
        o.step(40)
        ref = o.state()
        e = rel_pos_err(b.scene_state(s, full)["x"], ref["x"], sl[s].pos_mass[:, :3], sl[s].cell_size)
        assert e <= POS_TOL, f"scene {s}: position error vs FP64 oracle {e:.3e}"


def test_mixed_contact_batch_matches_scenes_alone():
    """Different grids, shape kinds and SDF-backed geometry in one batch (shape ids are global).
    The slicer scenes next to slicer-free ones exercise the per-particle choice between records
    carried from the previous G2P and records built from the stored state."""
    kinds = ["box", "sphere", "capsule", "trimesh", "lines", "arc", "dynamic_sphere", "effmass_sphere",
             "quad_slicer", "mesh_slicer"]
    sl = [scenes.contact_scene(k) for k in kinds]
    # the coupling scenes exchange forces through global shape ids: compare them too
    b = _check_against_alone(sl, 30, graph=False)
    force, torque = b.coupling()
    for s, sc in enumerate(sl):
        if sc.name not in ("dynamic_sphere", "effmass_sphere"):
            continue
        g = cb.DeviceScene(sc)
        g.step(30, graph=False)
        f1, t1 = g.coupling()
        sh = b.batch.shape_offset[s]  # shapes of scene s start at this merged shape index
        ids = sc.shapes.shape_ids
        np.testing.assert_allclose(force[b.batch.merged.shapes.shape_ids[sh:sh + len(ids)]], f1[ids], rtol=1e-3,
                                   atol=1e-6)


def _pb_pair(iterations=5):
    """A PB-MPM slab with the slicer blade inside it, and a PB-MPM cube without a slicer."""
    cut = scenes.pb_cutting(size=(0.12, 0.04, 0.12), cell=0.008, bounds_min=(-0.12, -0.1, -0.12),
                            bounds_max=(0.12, 0.1, 0.12), iterations=iterations)
    cut.shapes.position[1, :3] = (0.0, -0.01, 0.0)
    plain = scenes.cube_drop(solver=scenes.SOLVER_PB, dt=cut.dt)
    plain.mat_params[:, :2] = (1.0, 0.9)
    plain.iterations = iterations
    return plain, cut


def test_pb_batch_cut_masks_bit_exact():
    """PB-MPM with a quad-slicer scene next to plain scenes: masks match the single-scene run."""
    plain, cut = _pb_pair()
    sl = [plain, cut, plain]
    b = cb.DeviceBatch(sl)
    b.step(1, graph=False)
    masks = b.cut_masks()
    g = cb.DeviceScene(cut)
    g.step(1, graph=False)
    ref = g.cut_masks()
    np.testing.assert_array_equal(masks[b.batch.slice(1)], ref)
    assert ref.any(), "the slicer should cut some stencils"
    assert not masks[b.batch.slice(0)].any() and not masks[b.batch.slice(2)].any()


def test_pb_batch_matches_scenes_alone():
    """PB-MPM cutting amplifies rounding: after these 10 steps the reference's own float32 run
    departs from FP64 by 1.2e-2 of max(displacement, dx), and two float32 runs that differ only in
    the order of their sums by about 1e-4 to 1e-3; the batch is held to 20x the tolerances of the
    other batch tests (positions within 2e-3), still 6x inside the reference's own float32 drift."""
    plain, cut = _pb_pair()
    _check_against_alone([plain, cut], 10, tol_scale=20.0)


def test_standard_batch_matches_scenes_alone():
    sl = []
    for k, seed in enumerate((11, 12, 13)):
        sc = scenes.cube_drop(seed=seed, solver=scenes.SOLVER_STANDARD, dt=1e-4)
        sc.pos_mass[:, 0] += 0.1 * k
        sl.append(sc)
    _check_against_alone(sl, 40)


def test_batch_setters_apply_to_every_scene():
    sl = scenes.batched_scenes(num_scenes=2, nmin=1000, nmax=2000)
    b = cb.DeviceBatch(sl)
    b.solver.set_gravity((0.0, 0.0, 0.0))
    b.step(10)
    st = b.state()
    # no gravity, no initial velocity, nothing touching: the bodies stay at rest
    assert float(np.abs(st["v"]).max()) < 1e-6
