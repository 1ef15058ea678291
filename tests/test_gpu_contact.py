"""Contact, cutting and suturing geometry on the GPU against the CPU oracles.

Every geometry type of the reference's SDF set (include/geometry_utils/sdf.h:67-662) is exercised
by a falling cube: box, rotated non-uniformly scaled kinematic box, sphere, tilted plane, capsule,
arc and connected line segments (suturing: tangent-only response), a sampled triangle-mesh SDF,
quad and triangle-mesh slicers (cutting), and dynamic shapes with both contact models (coupling
force into the shape).  Slicer cut masks are compared bit for bit with the reference's own
predicate on identical positions.
"""
import numpy as np
import pytest

from conftest import cuda_available
from gpu_helpers import rel_pos_err

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

import crmpm_b200 as cb  # noqa: E402
import oracle_py as op  # noqa: E402
from crmpm_b200 import scenes  # noqa: E402

KINDS = ["box", "scaled_box", "sphere", "plane", "capsule", "arc", "lines", "trimesh", "quad_slicer", "mesh_slicer",
         "dynamic_sphere", "effmass_sphere"]


def _ref(sc):
    return op.RefOracle(sc) if op.ref_available() else op.PortOracle(sc, 32)


@pytest.mark.parametrize("kind", KINDS)
def test_contact_geometry_parity(kind):
    sc = scenes.contact_scene(kind)
    g = cb.DeviceScene(sc)
    o64 = op.PortOracle(sc, 64)
    r32 = _ref(sc)
    for o in (o64, r32):
        o.compute_initial_data()
    steps = 150
    g.step(steps)
    o64.step(steps)
    r32.step(steps)
    a, b, c = g.state(), o64.state(), r32.state()
    x0 = sc.pos_mass[:, :3]
    e_ref = rel_pos_err(c["x"], b["x"], x0, sc.cell_size)
    tol = max(1e-4, 2 * e_ref)
    assert rel_pos_err(a["x"], b["x"], x0, sc.cell_size) <= tol
    assert rel_pos_err(a["x"], c["x"], x0, sc.cell_size) <= tol
    assert float(np.abs(a["F"] - b["F"]).max()) <= max(1e-4, 2 * float(np.abs(c["F"] - b["F"]).max()))


@pytest.mark.parametrize("kind", ["quad_slicer", "mesh_slicer"])
def test_cut_masks_bitexact(kind):
    sc = scenes.contact_scene(kind)
    g = cb.DeviceScene(sc)
    r = _ref(sc)
    r.compute_initial_data()
    for _ in range(3):
        g.sync()
        x = g.pos[: sc.n].cpu().numpy()
        g.step(1, graph=False)
        got = g.cut_masks()
        if isinstance(r, op.RefOracle):
            r.pos[: sc.n] = x
        else:
            r.set_state(x=x[:, :3].astype(np.float64))
        exp = r.cut_masks()
        assert np.count_nonzero(exp) > 0
        np.testing.assert_array_equal(got, exp)
        g.step(20)


@pytest.mark.parametrize("kind", ["dynamic_sphere", "effmass_sphere"])
def test_dynamic_coupling_force(kind):
    sc = scenes.contact_scene(kind)
    g = cb.DeviceScene(sc)
    r = _ref(sc)
    r.compute_initial_data()
    g.step(100)
    r.step(100)
    f_gpu, t_gpu = g.coupling()
    sid = int(sc.shapes.shape_ids[0])
    if isinstance(r, op.RefOracle):
        f_ref, t_ref = r.coupling()
        f_ref, t_ref = f_ref[sid, :3], t_ref[sid, :3]
    else:
        c6 = r.coupling(sid)
        f_ref, t_ref = c6[:3], c6[3:]
    assert np.linalg.norm(f_ref) > 0.1
    np.testing.assert_allclose(f_gpu[sid, :3], f_ref, rtol=2e-3, atol=2e-3 * np.linalg.norm(f_ref))
    np.testing.assert_allclose(t_gpu[sid, :3], t_ref, rtol=5e-3, atol=5e-3 * max(np.linalg.norm(t_ref), 1e-3))


@pytest.mark.parametrize("kind", ["dynamic_sphere", "effmass_sphere"])
def test_deterministic_coupling_matches_atomic_coupling_and_oracle(kind):
    """CRB200_OPT_DETERMINISTIC_COUPLING sums the coupling momentum per grid block in a fixed order
    and then over blocks in ascending order: the totals must match the float-atomic totals (same
    terms, other order: within 1e-3 relative after 100 substeps of one run each, whose grids differ
    only by the P2G atomics' rounding) and the oracle within the bar of test_dynamic_coupling_force."""
    sc = scenes.contact_scene(kind)
    runs = {}
    for det in (0, 1):
        g = cb.DeviceScene(sc)
        g.solver.set_option(cb.OPT_DETERMINISTIC_COUPLING, det)
        g.step(100)
        runs[det] = g.coupling()
    sid = int(sc.shapes.shape_ids[0])
    (fa, ta), (fd, td) = runs[0], runs[1]
    assert np.linalg.norm(fa[sid, :3]) > 0.1
    np.testing.assert_allclose(fd[sid, :3], fa[sid, :3], rtol=1e-3, atol=1e-3 * np.linalg.norm(fa[sid, :3]))
    np.testing.assert_allclose(td[sid, :3], ta[sid, :3], rtol=1e-3, atol=1e-3 * max(np.linalg.norm(ta[sid, :3]), 1e-3))
    r = _ref(sc)
    r.compute_initial_data()
    r.step(100)
    if isinstance(r, op.RefOracle):
        f_ref, t_ref = r.coupling()
        f_ref, t_ref = f_ref[sid, :3], t_ref[sid, :3]
    else:
        c6 = r.coupling(sid)
        f_ref, t_ref = c6[:3], c6[3:]
    np.testing.assert_allclose(fd[sid, :3], f_ref, rtol=2e-3, atol=2e-3 * np.linalg.norm(f_ref))
    np.testing.assert_allclose(td[sid, :3], t_ref, rtol=5e-3, atol=5e-3 * max(np.linalg.norm(t_ref), 1e-3))


def test_deterministic_coupling_refused_on_batches():
    b = cb.DeviceBatch([scenes.contact_scene("dynamic_sphere"), scenes.contact_scene("box")])
    with pytest.raises(cb.CrmpmError, match="batch"):
        b.solver.set_option(cb.OPT_DETERMINISTIC_COUPLING, 1)


def test_pb_cutting_small():
    sc = scenes.pb_cutting(size=(0.12, 0.04, 0.12), cell=0.008, bounds_min=(-0.12, -0.1, -0.12),
                           bounds_max=(0.12, 0.1, 0.12), iterations=10)
    # put the blade inside the slab so that particles are actually cut
    sc.shapes.position[1, :3] = (0.0, -0.01, 0.0)
    g = cb.DeviceScene(sc)
    o64 = op.PortOracle(sc, 64)
    r32 = _ref(sc)
    for o in (o64, r32):
        o.compute_initial_data()
    steps = 10
    g.step(steps)
    o64.step(steps)
    r32.step(steps)
    a, b, c = g.state(), o64.state(), r32.state()
    x0 = sc.pos_mass[:, :3]
    e_ref = rel_pos_err(c["x"], b["x"], x0, sc.cell_size)
    tol = max(1e-4, 2 * e_ref)
    assert rel_pos_err(a["x"], b["x"], x0, sc.cell_size) <= tol
