"""The resident cell-ordered path (CRB200_OPT_RESIDENT, for single-scene MLS-MPM)
against the particle-id-ordered path of the same engine and against the FP64 oracle.

The two paths compute the same substep; they sum node contributions in different orders, so they
agree to float rounding, not bit for bit: positions within 1e-4 of max(displacement, dx),
velocities within 1e-3 of the velocity scale, F within 1e-4.  The cases cover what the resident
path adds: calls of different lengths, edits of the caller's buffers between calls, changes of the
particle set, mixed materials, slicers (cut masks kept per slot), coupling to dynamic shapes,
particles that drift far from the block they were grouped under (re-sort), and the exported F, C
and cut masks.
"""
import numpy as np
import pytest

from conftest import cuda_available
from gpu_helpers import rel_pos_err

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

import crmpm_b200 as cb  # noqa: E402
import oracle_py as op  # noqa: E402
from crmpm_b200 import scenes  # noqa: E402


def _scene(sc, resident):
    cb.build_library()
    g = cb.DeviceScene(sc)
    g.solver.set_option(cb.OPT_RESIDENT, 1 if resident else 0)
    return g


def _close(a, b, sc, what=""):
    x0 = sc.pos_mass[:, :3]
    e = rel_pos_err(a["x"], b["x"], x0, sc.cell_size)
    assert e <= 1e-4, f"{what}: positions differ by {e:.3e}"
    vscale = max(float(np.abs(b["v"]).max()), 1e-3)
    assert float(np.abs(a["v"] - b["v"]).max()) <= 1e-3 * vscale + 1e-6, what
    assert float(np.abs(a["F"] - b["F"]).max()) <= 1e-4, what
    cscale = max(float(np.abs(b["C"]).max()), 1e-3)
    assert float(np.abs(a["C"] - b["C"]).max()) <= 1e-3 * cscale, what
    np.testing.assert_array_equal(a["m"], b["m"])
    np.testing.assert_allclose(a["V0"], b["V0"], rtol=1e-6)


def _pair(sc, calls):
    """Both paths through the same sequence of step_many calls."""
    out = []
    for resident in (True, False):
        g = _scene(sc, resident)
        for n in calls:
            g.step(n)
        st = g.state()
        st["force"], st["torque"] = g.coupling()
        out.append(st)
    return out


@pytest.mark.parametrize("calls", [[200], [1, 1, 1, 7, 2, 40, 1]])
def test_cube_drop_matches_particle_order_path(calls):
    sc = scenes.cube_drop()
    a, b = _pair(sc, calls)
    _close(a, b, sc, f"calls {calls}")


def test_small_slab_matches_particle_order_path():
    sc = scenes.tissue_slab(size=(0.2, 0.06, 0.2), cell=0.01, bounds_min=(-0.15, -0.05, -0.15),
                            bounds_max=(0.15, 0.15, 0.15))
    a, b = _pair(sc, [100])
    _close(a, b, sc, "slab")


@pytest.mark.parametrize("kind", ["box", "sphere", "capsule", "arc", "lines", "trimesh", "scaled_box",
                                  "quad_slicer", "mesh_slicer", "dynamic_sphere", "effmass_sphere"])
def test_contact_scenes_match_particle_order_path(kind):
    sc = scenes.contact_scene(kind)
    a, b = _pair(sc, [30, 1, 29])
    _close(a, b, sc, kind)
    S = sc.shapes.shape_type.shape[0]
    for key in ("force", "torque"):
        scale = max(float(np.abs(b[key][:S]).max()), 1e-6)
        assert float(np.abs(a[key][:S] - b[key][:S]).max()) <= 1e-3 * scale, f"{kind} {key}"


def test_cut_masks_of_the_resident_slots_are_bitexact():
    """The resident path keeps each particle's slicer mask in its slot; exported in particle order
    they equal the oracle's masks of the positions the last substep started from."""
    sc = scenes.contact_scene("quad_slicer")
    g = _scene(sc, True)
    r = op.PortOracle(sc, 32)
    for _ in range(3):
        g.step(9)
        g.sync()
        x = g.pos[: sc.n].cpu().numpy()
        g.step(1, graph=False)
        got = g.cut_masks()
        r.set_state(x=x[:, :3].astype(np.float64))
        exp = r.cut_masks()
        assert np.count_nonzero(exp) > 0
        np.testing.assert_array_equal(got, exp)


def test_mixed_materials():
    """Two materials (and one co-rotational third): the resident path then reads each slot's
    material instead of the uniform one."""
    sc = scenes.cube_drop()
    lam2, mu2 = scenes.lame(4e4, 0.25)
    sc.mat_params[::2, :2] = (lam2, mu2)
    sc.mat_type[::3] = scenes.MAT_COROTATIONAL
    a, b = _pair(sc, [120])
    _close(a, b, sc, "mixed materials")
    o = op.PortOracle(sc, 64)
    o.compute_initial_data()
    o.step(120)
    assert rel_pos_err(a["x"], o.state()["x"], sc.pos_mass[:, :3], sc.cell_size) <= 1e-4


def test_edits_between_calls_are_honoured():
    """Velocities and positions written into the caller's buffers between calls take effect at the
    next call, on both paths alike."""
    import torch

    sc = scenes.cube_drop()
    out = []
    for resident in (True, False):
        g = _scene(sc, resident)
        g.step(50)
        g.sync()
        with torch.cuda.stream(g.stream):
            g.vel[: sc.n // 2, 0] += 0.5
            g.pos[sc.n // 2:, 1] += 0.003
        g.step(50)
        out.append(g.state())
    _close(out[0], out[1], sc, "edited buffers")


def test_particle_set_changes_between_calls():
    """Particles switched off (mask) and the active count lowered between calls: the resident
    slots are rebuilt; inactive particles never move."""
    import torch

    sc = scenes.cube_drop()
    out = []
    for resident in (True, False):
        g = _scene(sc, resident)
        g.step(40)
        g.sync()
        with torch.cuda.stream(g.stream):
            g.mask[::5] = 0
        g.solver.bind_active_mask(g.mask.data_ptr())
        g.step(30)
        g.solver.set_num_active_particles(sc.n - 100)
        g.sync()
        before = g.pos[sc.n - 100: sc.n, :3].cpu().numpy()
        g.step(30)
        st = g.state()
        after = g.pos[sc.n - 100: sc.n, :3].cpu().numpy()
        # the particles above the active count never move again
        np.testing.assert_array_equal(after, before, err_msg=f"resident={resident}")
        out.append(st)
    _close(out[0], out[1], sc, "particle set")


def test_drift_far_from_the_grouping_resorts():
    """A fast cube crossing several cells in one call (the slots' blocks are left behind and the
    slower paths take over) and again over several calls (re-sorts): same result as the
    particle-order path, and as close to FP64 as the reference's float32 run."""
    sc = scenes.cube_drop()
    sc.vel[:, :3] = (8.0, -6.0, 5.0)  # about five cells in x over the run
    a, b = _pair(sc, [150])
    _close(a, b, sc, "one call")
    c, _ = _pair(sc, [30] * 5)
    _close(c, b, sc, "five calls")
    o = op.PortOracle(sc, 64)
    o.compute_initial_data()
    o.step(150)
    x64 = o.state()["x"]
    r32 = op.RefOracle(sc) if op.ref_available() else op.PortOracle(sc, 32)
    r32.compute_initial_data()
    r32.step(150)
    x0 = sc.pos_mass[:, :3]
    tol = max(1e-4, 2.0 * rel_pos_err(r32.state()["x"], x64, x0, sc.cell_size))
    assert rel_pos_err(a["x"], x64, x0, sc.cell_size) <= tol
    assert rel_pos_err(c["x"], x64, x0, sc.cell_size) <= tol


def test_state_round_trip_and_phase_timing():
    """SetParticleState between resident calls replaces the resident F; the phase timing of the
    resident path counts one fused launch per substep after the first of each call."""
    sc = scenes.cube_drop()
    g = _scene(sc, True)
    g.step(20)
    st = g.state()
    ref = _scene(sc, False)
    ref.step(20)
    F = st["F"].copy()
    F[:, 0] *= 1.01
    for d in (g, ref):
        d.set_state(F=F)
        d.step(30)
    _close(g.state(), ref.state(), sc, "after SetParticleState")
    g.solver.set_option(cb.OPT_PHASE_TIMING, 1)
    g.solver.resident_kernel_time(reset=True)
    g.step(10)
    g.step(5)
    ms, launches = g.solver.resident_kernel_time(reset=True)
    g.solver.set_option(cb.OPT_PHASE_TIMING, 0)
    assert launches == 9 + 4 and ms > 0.0
