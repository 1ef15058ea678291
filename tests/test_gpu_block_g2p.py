"""The block-ordered MLS G2P (CRB200_OPT_BLOCK_G2P) against the id-ordered one.

Both compute each particle with the same source arithmetic; the block-ordered one gathers interior
stencils from a shared-memory node tile.  With deterministic substeps (no order-dependent float
sums anywhere) the two differ only by rounding, because the compiler may fuse multiply-adds
(weights, stencil offsets) differently in the two kernels.  One substep: every output within 1e-5
of its array's scale (1e-4 for C, a difference of nearly equal moments); after N substeps the
positions within 1e-5 of theirs.  A node read from the wrong place would move velocities by their
own size.  A particle given a non-finite position joins the scene's first cell, so the
block-ordered G2P reaches it as the id-ordered one does."""
import numpy as np
import pytest

from conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

import crmpm_b200 as cb  # noqa: E402
from crmpm_b200 import scenes  # noqa: E402


def _run(sc, steps, block):
    g = cb.DeviceScene(sc, compute_initial=False)
    g.solver.set_option(cb.OPT_DETERMINISTIC, 1)
    g.solver.set_option(cb.OPT_BLOCK_G2P, 1 if block else 0)
    g.compute_initial_data()
    g.step(steps)
    st = g.state()
    st["force"], st["torque"] = g.coupling()
    return st


def _nan_particle():
    sc = scenes.cube_drop()
    sc.pos_mass[7, :3] = np.nan
    return sc


CASES = {
    "cube": (lambda: scenes.cube_drop(), 100),
    "dense_cube": (lambda: scenes.cube_drop(ppc=27, side=0.3), 50),
    "dynamic_sphere": (lambda: scenes.contact_scene("dynamic_sphere"), 60),
    "small_slab": (lambda: scenes.tissue_slab(size=(0.3, 0.1, 0.3), bounds_min=(-0.2, -0.05, -0.2),
                                              bounds_max=(0.2, 0.2, 0.2)), 60),
    "nan_particle": (_nan_particle, 3),
}


def _close(a, b, k, tol, case):
    x, y = np.asarray(a[k], np.float64), np.asarray(b[k], np.float64)
    finite = np.isfinite(y)
    np.testing.assert_array_equal(np.isfinite(x), finite, err_msg=f"{case}: {k}")
    scale = max(float(np.abs(y[finite]).max(initial=0.0)), 1e-12)
    err = float(np.abs(x - y)[finite].max(initial=0.0))
    assert err <= tol * scale, f"{case}: {k}: {err:.3e} against scale {scale:.3e}"


@pytest.mark.parametrize("case", sorted(CASES))
def test_block_g2p_equals_id_order_g2p(case):
    make, steps = CASES[case]
    sc = make()
    a, b = _run(sc, 1, True), _run(sc, 1, False)
    for k, tol in (("x", 1e-5), ("v", 1e-5), ("F", 1e-5), ("C", 1e-4), ("force", 1e-5), ("torque", 1e-5)):
        _close(a, b, k, tol, case)
    a, b = _run(sc, steps, True), _run(sc, steps, False)
    _close(a, b, "x", 1e-5, case)
    if case == "nan_particle":
        # G2P clamps the non-finite position into the grid (fmin/fmax drop NaN operands)
        assert np.all(np.isfinite(a["x"][7]))
