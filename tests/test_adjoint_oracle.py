"""The FP64 host adjoint (oracle/adjoint_fp64.py) that the GPU adjoint is checked against.

Pinned two ways, on a cube hitting the ground (and, in the mixed scene, a kinematic spinning
sphere, a box and a tilted capsule): its forward substeps reproduce the FP64 restatement of the
reference (PortOracle, double) to rounding, and its gradients with respect to Young's modulus,
Poisson's ratio and the initial velocity match central finite differences of its own forward
within 1e-5 relative.
"""
import numpy as np
import pytest

import oracle_py as op
from adjoint_fp64 import Fp64Adjoint, lame, lame_grad
from crmpm_b200 import scenes

STEPS = 30
CAPS = (10, 20, 30)


@pytest.mark.parametrize("kind", ["plane", "mixed", "effmass"])
def test_fp64_forward_matches_oracle(kind):
    sc = scenes.adjoint_scene(kind)
    a = Fp64Adjoint(sc)
    xs = a.forward(sc.mat_params[:, 0], sc.mat_params[:, 1], sc.vel[:, :3], STEPS)
    o = op.PortOracle(sc, 64)
    o.compute_initial_data()
    o.step(STEPS)
    st = o.state()
    x, v, F, C = a.tape[-1]
    assert xs[-1][:, 1].min() < 0.005, "the cube should reach the ground"
    # plane only: equal to double rounding; with the rotated shapes the two codes rotate
    # differently (quaternion formula vs matrix), which contact amplifies to ~1e-8
    tol = 1e-12 if kind == "plane" else 1e-7
    np.testing.assert_allclose(x, st["x"], atol=tol)
    np.testing.assert_allclose(v, st["v"], atol=tol)
    np.testing.assert_allclose(F.transpose(0, 2, 1).reshape(-1, 9), st["F"], atol=tol)
    np.testing.assert_allclose(C.transpose(0, 2, 1).reshape(-1, 9), st["C"], atol=tol)
    np.testing.assert_allclose(a.V0, st["V0"], rtol=1e-12)


@pytest.mark.parametrize("kind", ["plane", "mixed", "effmass"])
def test_fp64_adjoint_matches_central_differences(kind):
    sc = scenes.adjoint_scene(kind)
    n = sc.n
    E, nu = 2e4, 0.35
    v0 = sc.vel[:, :3].astype(np.float64)
    rng = np.random.default_rng(7)
    a = Fp64Adjoint(sc)
    lam, mu = lame(E, nu)
    xs = a.forward(np.full(n, lam), np.full(n, mu), v0, STEPS)
    tgt = {t: xs[t - 1] + rng.normal(0.0, 1e-3, xs[t - 1].shape) for t in CAPS}

    def loss(E_, nu_, dv):
        l_, m_ = lame(E_, nu_)
        b = Fp64Adjoint(sc)
        ys = b.forward(np.full(n, l_), np.full(n, m_), v0 + dv, STEPS)
        return sum(((ys[t - 1] - tgt[t]) ** 2).mean() for t in CAPS)

    g = a.backward({t: 2.0 * (xs[t - 1] - tgt[t]) / (3 * n) for t in CAPS})
    (dlE, dlnu), (dmE, dmnu) = lame_grad(E, nu)
    gE = float((g["g_lam"] * dlE + g["g_mu"] * dmE).sum())
    gnu = float((g["g_lam"] * dlnu + g["g_mu"] * dmnu).sum())
    gv = g["g_v0"].sum(0)
    h = 1e-5
    fE = (loss(E * (1 + h), nu, 0.0) - loss(E * (1 - h), nu, 0.0)) / (2 * E * h)
    fnu = (loss(E, nu * (1 + h), 0.0) - loss(E, nu * (1 - h), 0.0)) / (2 * nu * h)
    assert abs(gE - fE) <= 1e-5 * abs(fE), (gE, fE)
    assert abs(gnu - fnu) <= 1e-5 * abs(fnu), (gnu, fnu)
    for k in range(3):
        dv = np.zeros(3)
        dv[k] = 1e-5
        fv = (loss(E, nu, dv) - loss(E, nu, -dv)) / 2e-5
        assert abs(gv[k] - fv) <= 1e-5 * max(abs(fv), 1e-3 * np.abs(gv).max()), (k, gv[k], fv)
