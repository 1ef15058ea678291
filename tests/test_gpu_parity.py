"""Parity of the sm_100a engine (through the C ABI) with the CPU oracles.

Tolerances (float32 kernels vs the FP64 oracle, and vs the reference's own float32 arithmetic):
positions within max(1e-4, 2 x the reference float32 run's own deviation from FP64) of
max(displacement, dx) after the full run; velocities within 1e-3 of the velocity scale (or twice
the reference's own deviation); deformation gradients within 1e-4 absolute (same rule).  Integer
outputs (cell keys, the sort permutation, slicer cut masks) must match bit for bit on identical
float inputs.
"""
import numpy as np
import pytest

from conftest import cuda_available
from gpu_helpers import block_keys, canonical_permutation, rel_pos_err

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

import crmpm_b200 as cb  # noqa: E402
import oracle_py as op  # noqa: E402
from crmpm_b200 import scenes  # noqa: E402

POS_TOL = 1e-4
F_TOL = 1e-4


def _gpu(sc, **kw):
    cb.build_library()
    return cb.DeviceScene(sc, **kw)


def _compare(sc, steps, pos_tol=POS_TOL, f_tol=F_TOL, v_tol=1e-3):
    """GPU vs the FP64 oracle and vs the reference's float32 arithmetic.

    Contact-heavy scenes are sensitive: the reference's own float32 run drifts from FP64 by more
    than 1e-4.  The GPU must then stay within twice that drift of FP64 (and of the float32 run).
    """
    g = _gpu(sc)
    o64 = op.PortOracle(sc, 64)
    o64.compute_initial_data()
    r32 = op.RefOracle(sc) if op.ref_available() else op.PortOracle(sc, 32)
    r32.compute_initial_data()
    g.step(steps)
    o64.step(steps)
    r32.step(steps)
    a, b, c = g.state(), o64.state(), r32.state()
    x0 = sc.pos_mass[:, :3]
    e_ref = rel_pos_err(c["x"], b["x"], x0, sc.cell_size)
    tol = max(pos_tol, 2.0 * e_ref)
    e64 = rel_pos_err(a["x"], b["x"], x0, sc.cell_size)
    e32 = rel_pos_err(a["x"], c["x"], x0, sc.cell_size)
    assert e64 <= tol, f"position error vs FP64 {e64:.3e} (reference float32 vs FP64: {e_ref:.3e})"
    assert e32 <= tol, f"position error vs reference float32 {e32:.3e} (reference float32 vs FP64: {e_ref:.3e})"
    vscale = max(float(np.abs(b["v"]).max()), 1e-3)
    dv_ref = float(np.abs(c["v"] - b["v"]).max())
    assert float(np.abs(a["v"] - b["v"]).max()) <= max(v_tol * vscale, 2.0 * dv_ref) + 1e-6
    df_ref = float(np.abs(c["F"] - b["F"]).max())
    assert float(np.abs(a["F"] - b["F"]).max()) <= max(f_tol, 2.0 * df_ref)
    np.testing.assert_allclose(a["V0"], b["V0"], rtol=1e-5)
    return a, b


def test_initial_volume_matches_reference_order_oracle():
    sc = scenes.cube_drop()
    g = _gpu(sc)
    o = op.PortOracle(sc, 32)
    o.compute_initial_data()
    a, b = g.state(), o.state()
    np.testing.assert_allclose(a["V0"], b["V0"], rtol=2e-6)
    np.testing.assert_array_equal(a["F"], np.tile(np.eye(3).T.ravel(), (sc.n, 1)).astype(np.float32))


def test_mls_cube_drop_500_substeps():
    """The reference's own CPU-runnable case: 4096-particle Neo-Hookean cube onto a plane."""
    _compare(scenes.cube_drop(), 500)


@pytest.mark.parametrize("material", [scenes.MAT_COROTATIONAL, scenes.MAT_LINEAR_ELASTIC])
def test_mls_materials(material):
    _compare(scenes.cube_drop(material=material), 200)


def test_standard_mpm_cube():
    _compare(scenes.cube_drop(solver=scenes.SOLVER_STANDARD, dt=1e-4), 200)


def test_pb_mpm_cube():
    sc = scenes.cube_drop(solver=scenes.SOLVER_PB, dt=0.002)
    sc.mat_params[:, :2] = (1.0, 0.9)
    sc.iterations = 10
    _compare(sc, 30, f_tol=2e-4)


def test_sort_keys_and_permutation_bitexact():
    """CrB200SolverCopySortState sorts the current positions: cell keys and the canonical
    permutation (by key, ties by particle id) bit for bit against numpy."""
    sc = scenes.cube_drop()
    g = _gpu(sc)
    for _ in range(3):
        g.step(1, graph=False)
        g.sync()
        x_now = g.pos[: sc.n, :3].cpu().numpy()
        keys, ids = g.sort_state()
        exp = block_keys(sc, x_now)
        np.testing.assert_array_equal(keys, exp)
        np.testing.assert_array_equal(ids, canonical_permutation(exp, sc.mask.astype(bool)))
        g.step(40)


def test_inactive_particles_are_skipped():
    sc = scenes.cube_drop()
    sc.mask[::7] = 0
    a, b = _compare(sc, 100)
    # inactive particles never move
    np.testing.assert_array_equal(a["x"][::7], sc.pos_mass[::7, :3])


def test_tissue_slab_small_with_probe():
    sc = scenes.tissue_slab(size=(0.2, 0.06, 0.2), cell=0.01, bounds_min=(-0.15, -0.05, -0.15),
                            bounds_max=(0.15, 0.15, 0.15))
    _compare(sc, 100)


def test_determinism_run_to_run():
    sc = scenes.cube_drop()
    runs = []
    for _ in range(2):
        g = _gpu(sc)
        g.step(50)
        runs.append(g.state())
    for k in ("x", "v", "F", "C"):
        # float atomics make the order of node sums vary between runs; differences stay at rounding level
        assert float(np.abs(runs[0][k] - runs[1][k]).max()) <= 1e-5


def test_status_reports_nan_velocity():
    sc = scenes.cube_drop()
    sc.vel[10, 0] = np.nan
    g = _gpu(sc)
    g.step(2, graph=False)
    st = g.solver.status()
    assert st & cb.STATUS_NAN_STATE
    g.solver.clear_status()
    assert g.solver.status() == 0


def test_advance_sync_and_async_match_the_oracle():
    """Scene-style advance (CrB200SolverAdvance and its asynchronous form) runs the reference's
    float substep count and reads back positions and velocities; three frames of each, the async
    one alternating two host buffer pairs, must agree with each other and with the FP64 oracle."""
    import torch

    sc = scenes.cube_drop()
    frame = float(np.float32(sc.dt) * 7) * 0.999  # 7 substeps by the float accumulation
    out = {}
    for mode in ("sync", "async"):
        g = _gpu(sc)
        bufs = [(torch.empty((g.num_max, 4), dtype=torch.float32, pin_memory=True),
                 torch.empty((g.num_max, 4), dtype=torch.float32, pin_memory=True)) for _ in range(2)]
        total = 0
        for k in range(3):
            hx, hv = bufs[k & 1]
            if mode == "sync":
                total += g.solver.advance(frame, hx.data_ptr(), hv.data_ptr())
            else:
                total += g.solver.advance_async(frame, hx.data_ptr(), hv.data_ptr())
        g.solver.fetch_results()
        assert total == 21
        out[mode] = (bufs[0][0][: sc.n].numpy().copy(), bufs[0][1][: sc.n].numpy().copy())  # frame 3
    o = op.PortOracle(sc, 64)
    o.compute_initial_data()
    o.step(21)
    ref = o.state()
    x0 = sc.pos_mass[:, :3]
    for mode, (hx, hv) in out.items():
        assert rel_pos_err(hx[:, :3], ref["x"], x0, sc.cell_size) <= POS_TOL, mode
        np.testing.assert_array_equal(hx[:, 3], sc.pos_mass[:, 3])  # masses travel with positions
    np.testing.assert_allclose(out["sync"][0][:, :3], out["async"][0][:, :3], atol=1e-6)


SOLVER_ADAPTER_CHECK = __import__("os").path.join(
    __import__("os").path.dirname(__import__("os").path.dirname(__import__("os").path.abspath(__file__))),
    "oracle", "_ref", "solver_adapter_check")


@pytest.mark.skipif(not __import__("os").path.exists(SOLVER_ADAPTER_CHECK),
                    reason="oracle/_ref/solver_adapter_check not built")
@pytest.mark.parametrize("solver", [scenes.SOLVER_MLS, scenes.SOLVER_PB, scenes.SOLVER_STANDARD])
def test_reference_side_solver_adapter_runs_the_engine(solver, tmp_path):
    """The drop-in solver (adapter/gpu_b200_mpm_solver.h) driven through the reference's own
    MpmSolverBase / MpmSolverGpu members, in the factory's and the scene's order, gives the
    engine's result (float atomics aside) and stays within the parity tolerance of the oracle."""
    import subprocess

    dt = {scenes.SOLVER_MLS: 2e-4, scenes.SOLVER_PB: 2e-3, scenes.SOLVER_STANDARD: 1e-4}[solver]
    sc = scenes.cube_drop(solver=solver, dt=dt)
    if solver == scenes.SOLVER_PB:
        sc.mat_params[:, :2] = (1.0, 0.9)
    steps = 10 if solver == scenes.SOLVER_PB else 100
    path, out = tmp_path / "scene.bin", tmp_path / "out.bin"
    with open(path, "wb") as f:
        np.asarray([sc.n, solver], np.int32).tofile(f)
        np.asarray([sc.cell_size, sc.dt, *sc.grid_min, *sc.grid_max, *sc.gravity, 0.3, 1.0], np.float32).tofile(f)
        for a in (sc.pos_mass, sc.vel, sc.mat_params):
            np.ascontiguousarray(a, np.float32).tofile(f)
        np.ascontiguousarray(sc.mat_type, np.int32).tofile(f)
    r = subprocess.run([SOLVER_ADAPTER_CHECK, str(path), str(steps), str(out)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    res = np.fromfile(out, np.float32).reshape(2, sc.n, 4)
    # the PB-MPM adapter keeps the reference's default of 10 solver iterations (setSolverIterations)
    sc.iterations = 10
    g = _gpu(sc)
    g.step(steps)
    a = g.state()
    x0 = sc.pos_mass[:, :3]
    assert rel_pos_err(res[0, :, :3], a["x"], x0, sc.cell_size) <= 1e-4
    o = op.PortOracle(sc, 64)
    o.compute_initial_data()
    o.step(steps)
    tol = 2e-3 if solver == scenes.SOLVER_PB else 1e-4
    assert rel_pos_err(res[0, :, :3], o.state()["x"], x0, sc.cell_size) <= tol
