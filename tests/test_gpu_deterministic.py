"""Deterministic substeps (CRB200_OPT_DETERMINISTIC): P2G stores whole block tiles and the grid
update sums each node's tiles in a fixed order; the coupling momentum is reduced in a fixed order
(single scenes; batches keep the coupling atomics and reproduce the particle state).
Two runs from the same state must agree bit for bit (the ordinary path sums with float atomics in
arrival order, as the reference does, and does not), and a deterministic run must stay within the
parity tolerance of the ordinary run and of the FP64 oracle."""
import numpy as np
import pytest

from conftest import cuda_available
from gpu_helpers import rel_pos_err

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

import crmpm_b200 as cb  # noqa: E402
import oracle_py as op  # noqa: E402
from crmpm_b200 import scenes  # noqa: E402


def _pb_cut():
    sc = scenes.pb_cutting(size=(0.12, 0.04, 0.12), cell=0.008, bounds_min=(-0.12, -0.1, -0.12),
                           bounds_max=(0.12, 0.1, 0.12), iterations=10)
    sc.shapes.position[1, :3] = (0.0, -0.01, 0.0)
    return sc


CASES = {
    "mls_cube": (lambda: scenes.cube_drop(), 200),
    # 27 particles per cell: every cell overflows the 9 a cell thread accumulates
    "mls_dense": (lambda: scenes.cube_drop(ppc=27, side=0.3), 100),
    "dynamic_sphere": (lambda: scenes.contact_scene("dynamic_sphere"), 100),
    "effmass_sphere": (lambda: scenes.contact_scene("effmass_sphere"), 100),
    "pb_cutting": (_pb_cut, 5),
    "standard_cube": (lambda: scenes.cube_drop(solver=scenes.SOLVER_STANDARD, dt=1e-4), 200),
}


def _run(sc, steps, det):
    # the option goes on before the initial data: their node masses are summed deterministically too
    g = cb.DeviceScene(sc, compute_initial=False)
    if det:
        g.solver.set_option(cb.OPT_DETERMINISTIC, 1)
    g.compute_initial_data()
    g.step(steps)
    st = g.state()
    f, t = g.coupling()
    return st, f, t


@pytest.mark.parametrize("case", sorted(CASES))
def test_deterministic_runs_repeat_bit_for_bit(case):
    make, steps = CASES[case]
    sc = make()
    a, fa, ta = _run(sc, steps, True)
    b, fb, tb = _run(sc, steps, True)
    for k in ("x", "v", "F", "C"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"{case}: {k} differs between two deterministic runs")
    np.testing.assert_array_equal(fa, fb)
    np.testing.assert_array_equal(ta, tb)
    # the ordinary (atomic) path: same physics within the parity tolerance
    c, fc, tc = _run(sc, steps, False)
    tol = 2e-3 if case == "pb_cutting" else 1e-4  # PB-MPM cutting amplifies rounding (see test_gpu_batch)
    assert rel_pos_err(a["x"], c["x"], sc.pos_mass[:, :3], sc.cell_size) <= tol


def test_deterministic_mls_cube_matches_fp64_oracle():
    sc = scenes.cube_drop()
    a, _, _ = _run(sc, 200, True)
    o = op.PortOracle(sc, 64)
    o.compute_initial_data()
    o.step(200)
    assert rel_pos_err(a["x"], o.state()["x"], sc.pos_mass[:, :3], sc.cell_size) <= 1e-4


def _batch_run(sl, steps, det):
    b = cb.DeviceBatch(sl, compute_initial=False)
    if det:
        b.solver.set_option(cb.OPT_DETERMINISTIC, 1)
    b.compute_initial_data()
    b.step(steps)
    return b, b.state()


def test_deterministic_batch_repeats_bit_for_bit():
    """A batch in deterministic mode: two runs give the same particle state bit for bit, and each
    scene stays within the parity tolerance of the ordinary (atomic) batch run."""
    sl = scenes.batched_scenes(num_scenes=8, nmin=2000, nmax=8000)
    steps = 60
    b1, a = _batch_run(sl, steps, True)
    _, c = _batch_run(sl, steps, True)
    for k in ("x", "v", "F", "C"):
        np.testing.assert_array_equal(a[k], c[k], err_msg=f"batch {k} differs between two deterministic runs")
    _, o = _batch_run(sl, steps, False)
    for s, sc in enumerate(sl):
        got, ref = b1.scene_state(s, a), b1.scene_state(s, o)
        assert rel_pos_err(got["x"], ref["x"], sc.pos_mass[:, :3], sc.cell_size) <= 1e-4, f"scene {s}"


@pytest.mark.parametrize("case", ["mls_cube", "dynamic_sphere"])
def test_call_lengths_give_the_same_state_bit_for_bit(case):
    """Within a call, the substeps but the last leave the velocity and C to the P2G record their
    G2P writes for the next substep; the call's last substep writes them.  In deterministic mode
    one call of n substeps, n calls of one and calls of mixed lengths must give the same state
    bit for bit."""
    make, _ = CASES[case]
    sc = make()
    out = []
    for calls in ([60], [1] * 60, [7, 1, 23, 2, 27]):
        g = cb.DeviceScene(sc, compute_initial=False)
        g.solver.set_option(cb.OPT_DETERMINISTIC, 1)
        g.compute_initial_data()
        for n in calls:
            g.step(n)
        st = g.state()
        st["force"], st["torque"] = g.coupling()
        out.append(st)
    for other in out[1:]:
        for k in ("x", "v", "F", "C", "force", "torque"):
            np.testing.assert_array_equal(out[0][k], other[k], err_msg=f"{case}: {k}")
