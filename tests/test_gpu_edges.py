"""Edge cases of the substep engine and of the SDF builder on the GPU: no active particle, one
particle, particles leaving the domain, a particle exactly on a block boundary, meshes of one
triangle and meshes with a zero-area triangle.  Each is checked against the CPU oracle (or the
SDF restatement) where there is a result to compare."""
import numpy as np
import pytest

from conftest import cuda_available
from gpu_helpers import rel_pos_err

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

import crmpm_b200 as cb  # noqa: E402
import oracle_py as op  # noqa: E402
from crmpm_b200 import meshes, scenes  # noqa: E402


def _oracle(sc, steps):
    o = op.PortOracle(sc, 64)
    o.compute_initial_data()
    o.step(steps)
    return o.state()


def test_no_active_particle_steps_and_changes_nothing():
    sc = scenes.cube_drop()
    sc.mask[:] = 0
    g = cb.DeviceScene(sc)
    g.step(20)
    st = g.state()
    np.testing.assert_array_equal(st["x"], sc.pos_mass[:, :3])
    np.testing.assert_array_equal(st["v"], sc.vel[:, :3])
    assert g.solver.status() == 0


def test_single_particle_free_fall_matches_oracle():
    sc = scenes.cube_drop()
    keep = slice(0, 1)
    for k in ("pos_mass", "vel", "mat_params", "mat_type", "mask"):
        setattr(sc, k, np.ascontiguousarray(getattr(sc, k)[keep]))
    sc.pos_mass[0, :3] = (0.013, 0.61, -0.027)
    g = cb.DeviceScene(sc)
    g.step(60)
    got = g.state()
    ref = _oracle(sc, 60)
    assert rel_pos_err(got["x"], ref["x"], sc.pos_mass[:, :3], sc.cell_size) <= 1e-4
    np.testing.assert_allclose(got["v"], ref["v"], rtol=1e-4, atol=1e-6)
    assert float(got["v"][0, 1]) < 0.0  # falling


def test_particles_on_block_boundaries_match_oracle():
    """Particles placed exactly on cell and 4x4x4-block boundaries (integer multiples of dx from
    the grid origin): the cell key and base node are decided by truncation exactly as the
    reference's, and the run matches the oracle."""
    sc = scenes.cube_drop()
    dx = np.float32(sc.cell_size)
    gmin = sc.grid_min.astype(np.float32)
    pts = np.array([[24, 28, 24], [25, 29, 25], [28, 32, 28], [32, 30, 20], [20, 33, 31]], np.float32)
    sc.pos_mass[:5, :3] = gmin + pts * dx
    g = cb.DeviceScene(sc)
    g.step(50)
    got = g.state()
    ref = _oracle(sc, 50)
    assert rel_pos_err(got["x"], ref["x"], sc.pos_mass[:, :3], sc.cell_size) <= 1e-4


def test_particles_leaving_the_domain_are_clamped():
    """A particle shot out of the grid: positions stay clamped to the grid bounds as the
    reference clamps them (math_helpers.h:250-255), and the rest of the body is unaffected
    (matches the oracle)."""
    sc = scenes.cube_drop()
    sc.vel[3, :3] = (0.0, 400.0, 0.0)  # leaves through the top within a few substeps
    g = cb.DeviceScene(sc)
    g.step(30, graph=False)
    got = g.state()
    assert np.all(got["x"] <= sc.grid_max + 1e-6) and np.all(got["x"] >= sc.grid_min - 1e-6)
    ref = _oracle(sc, 30)
    others = np.ones(sc.n, bool)
    others[3] = False
    assert rel_pos_err(got["x"][others], ref["x"][others], sc.pos_mass[others, :3], sc.cell_size) <= 1e-4


def _sdf_vs_restatement(P, T, cell, fatten, slicer=False):
    cb.build_library()
    g = cb.build_sdf(P, T, cell, fatten, slicer=slicer)
    import torch

    torch.cuda.synchronize()
    _, _, _, ref = op.port_sdf(P, T, cell, fatten, slicer=slicer)
    got = g.host()
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    np.testing.assert_array_equal(got[~np.isnan(ref)], ref[~np.isnan(ref)])
    return got


def test_sdf_of_one_triangle():
    P = np.array([[0.1, 0.0, 0.0], [0.3, 0.05, 0.0], [0.15, 0.2, 0.02]], np.float32)
    T = np.array([[0, 1, 2]], np.uint32)
    got = _sdf_vs_restatement(P, T, 0.02, 0.03)
    assert np.all(got[:, 3] >= 0.0)  # an open sheet encloses nothing
    _sdf_vs_restatement(P, T, 0.02, 0.03, slicer=True)


def test_sdf_with_a_zero_area_triangle():
    P, T = meshes.icosphere(0.2, 1)
    P = np.vstack([P, P[:1]])  # a duplicate of vertex 0
    T = np.vstack([T, [[0, len(P) - 1, 1]]]).astype(np.uint32)  # degenerate: two equal corners
    _sdf_vs_restatement(P, T, 0.03, 0.05)


def test_sdf_rejects_a_single_node_axis():
    P = np.array([[0.0, 0.0, 0.0], [0.5, 0.0, 0.0], [0.0, 0.5, 0.0]], np.float32)
    T = np.array([[0, 1, 2]], np.uint32)
    d = cb.sdf_desc(P, T, 10.0)  # a cell far larger than the mesh: one node per axis
    assert min(d.sdfDimension) < 2
    with pytest.raises(cb.CrmpmError, match="at least 2"):
        cb.build_sdf(P, T, 10.0)
