"""Pins the CPU restatement (oracle/mpm_oracle.cpp) against the reference's own arithmetic.

``RefOracle`` runs CRESSim-MPM's header-only algorithms compiled for the host; ``PortOracle`` is
this repository's independent restatement.  In float mode the restatement follows the reference's
operation order, so everything except the SVD-based PB-MPM constraint must agree bit for bit.
When the reference sources are absent (GPU box) the committed golden fixtures stand in for it
(tests/test_golden.py).
"""
import numpy as np
import pytest

import oracle_py as op
from crmpm_b200 import scenes

pytestmark = pytest.mark.skipif(not op.ref_available(), reason="reference driver not built (no reference sources)")


def _run_both(sc, steps, idx=None):
    r = op.RefOracle(sc)
    p = op.PortOracle(sc, 32)
    r.compute_initial_data(idx)
    p.compute_initial_data(idx)
    r.step(steps)
    p.step(steps)
    return r.state(), p.state()


@pytest.mark.parametrize("material", [scenes.MAT_NEOHOOKEAN, scenes.MAT_COROTATIONAL, scenes.MAT_LINEAR_ELASTIC])
def test_mls_cube_bitexact(material):
    sc = scenes.cube_drop(material=material)
    a, b = _run_both(sc, 200)
    for k in ("x", "v", "F", "C", "V0"):
        np.testing.assert_array_equal(a[k], b[k].astype(np.float32), err_msg=k)


def test_standard_cube_bitexact():
    sc = scenes.cube_drop(solver=scenes.SOLVER_STANDARD, dt=1e-4)
    a, b = _run_both(sc, 100)
    for k in ("x", "v", "F", "V0"):
        np.testing.assert_array_equal(a[k], b[k].astype(np.float32), err_msg=k)


def test_pb_cube_close():
    # PB-MPM goes through the 3x3 SVD, where the restatement uses its own rotations.
    sc = scenes.cube_drop(solver=scenes.SOLVER_PB, dt=0.002)
    sc.mat_params[:, :2] = (1.0, 0.9)
    sc.iterations = 5
    a, b = _run_both(sc, 20)
    scale = np.abs(a["x"] - sc.pos_mass[:, :3]).max()
    assert np.abs(a["x"] - b["x"]).max() <= 1e-4 * max(scale, sc.cell_size)
    assert np.abs(a["F"] - b["F"]).max() <= 1e-4


@pytest.mark.parametrize("spread,tol_max", [(0.1, 5e-5), (1.0, 2e-2)])
def test_svd_matches_reference(spread, tol_max):
    # The reference's fixed 4-sweep approximate Jacobi SVD agrees with an exact SVD to ~3e-7 in
    # the median; its worst case grows with the spread of the matrix (1e-5 near the identity,
    # where deformation gradients live, 1e-2 on arbitrary matrices).  The tolerances follow that.
    rng = np.random.default_rng(3)
    A = (rng.normal(size=(500, 9)) * spread).astype(np.float32)
    A[:, [0, 4, 8]] += 1.0
    U, Vt, S = op.ref_svd3(A)
    Up, Vp, Sp = op.port_svd3(A, 64)
    assert np.abs(Sp - S).max() <= tol_max
    # The reference factors the transpose of its argument (svd3.h:1271-1274): u*vt = V U^T of A.
    R_ref = U.reshape(-1, 3, 3).transpose(0, 2, 1) @ Vt.reshape(-1, 3, 3).transpose(0, 2, 1)
    Vm = Vp.reshape(-1, 3, 3).transpose(0, 2, 1)
    Um = Up.reshape(-1, 3, 3).transpose(0, 2, 1)
    err = np.abs(Vm @ Um.transpose(0, 2, 1) - R_ref).max(axis=(1, 2))
    assert np.median(err) <= 1e-6
    assert err.max() <= tol_max


def test_svd_known_answer_from_reference_test():
    # The matrix of the reference's SVD printout test (tests/test_svd/main.cpp:36).
    A = np.array([[1, 2, 5, 3, 1, 4, 2, 9, 3]], np.float32)
    U, Vt, S = op.ref_svd3(A)
    Up, Vp, Sp = op.port_svd3(A, 64)
    np.testing.assert_allclose(np.abs(Sp), np.abs(S), rtol=1e-5)
    M = A.reshape(3, 3).T
    rec = Up.reshape(3, 3).T @ np.diag(Sp[0]) @ Vp.reshape(3, 3)
    np.testing.assert_allclose(rec, M, atol=1e-9)
