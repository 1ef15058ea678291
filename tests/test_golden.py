"""The CPU restatement against fixtures produced by the reference's own arithmetic.

tests/golden/*.npz were generated by tests/golden/make_golden.py from oracle/_ref (the reference's
header-only algorithms compiled for the host).  Each fixture holds its scene, so these tests need
neither the reference sources nor a GPU.  MLS and standard MPM and every contact geometry must be
bit-identical; PB-MPM differs only through the SVD and is held to 1e-5 of dx.
"""
import glob
import os

import numpy as np
import pytest

import oracle_py as op
from crmpm_b200 import scenes

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def scene_from(z):
    st = scenes.ShapeTable(*[z["sh_" + k] for k in (
        "shape_type", "geom_idx", "position", "rotation", "inv_scale", "lin_vel", "ang_vel", "com_inv_mass", "inertia0",
        "inertia1", "force", "torque", "params0", "geom_type", "geom_params", "sdf_dims", "sdf_lbcs", "sdf_data",
        "shape_ids")])
    st.force = st.force.copy()
    st.torque = st.torque.copy()
    return scenes.Scene(int(z["solver_type"]), z["grid_min"], z["grid_max"], float(z["cell_size"]), float(z["dt"]),
                        z["gravity"], int(z["iterations"]), int(z["contact_model"]), z["pos_mass"].copy(), z["vel"].copy(),
                        z["mat_params"].copy(), z["mat_type"].copy(), z["mask"].copy(), st)


CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLD, "*.npz"))
               if not os.path.basename(p).startswith(("svd3", "sdf_queries", "meshsdf_")))


def test_fixtures_present():
    assert len(CASES) >= 10


@pytest.mark.parametrize("case", CASES)
def test_port_matches_reference_fixture(case):
    z = np.load(os.path.join(GOLD, case + ".npz"))
    sc = scene_from(z)
    o = op.PortOracle(sc, 32)
    o.compute_initial_data()
    np.testing.assert_array_equal(o.state()["V0"].astype(np.float32), z["V0_init"])
    np.testing.assert_array_equal(o.cut_masks(), z["masks0"])
    o.step(int(z["steps"]))
    s = o.state()
    if sc.solver_type == scenes.SOLVER_PB:
        assert np.abs(s["x"] - z["x"]).max() <= 1e-5 * sc.cell_size
        assert np.abs(s["F"] - z["F"]).max() <= 1e-4
        return
    for k in ("x", "v", "F", "C", "V0"):
        np.testing.assert_array_equal(s[k].astype(np.float32), z[k], err_msg=k)
    if sc.contact_model == 1 or "dynamic" in case:
        sid = int(sc.shapes.shape_ids[0])
        c6 = o.coupling(sid)
        np.testing.assert_allclose(c6[:3], z["force"][sid, :3], rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(c6[3:], z["torque"][sid, :3], rtol=1e-6, atol=1e-7)


def test_sdf_queries_bitexact():
    z = np.load(os.path.join(GOLD, "sdf_queries.npz"))
    kinds = sorted({k.split("_gtype")[0] for k in z.files if k.endswith("_gtype")})
    assert len(kinds) == 9
    for kind in kinds:
        st = scenes.ShapeTable.empty()
        st.sdf_dims, st.sdf_lbcs, st.sdf_data = z[f"{kind}_sdf_dims"], z[f"{kind}_sdf_lbcs"], z[f"{kind}_sdf_data"]
        out, tan, spine = op.sdf_query("port", int(z[f"{kind}_gtype"]), z[f"{kind}_params"], st, z[f"{kind}_pts"], prec=32)
        np.testing.assert_array_equal(out.astype(np.float32), z[f"{kind}_out"], err_msg=kind)
        np.testing.assert_array_equal(spine, z[f"{kind}_spine"], err_msg=kind)
        if kind in ("arc", "lines"):
            np.testing.assert_array_equal(tan[:, :3].astype(np.float32), z[f"{kind}_tan"][:, :3], err_msg=kind)


def test_svd_against_reference_fixture():
    z = np.load(os.path.join(GOLD, "svd3.npz"))
    U, V, S = op.port_svd3(z["A"], 64)
    np.testing.assert_allclose(np.abs(S), np.abs(z["S"]), rtol=1e-5, atol=1e-5)
    R_ref = z["U"].reshape(-1, 3, 3).transpose(0, 2, 1) @ z["Vt"].reshape(-1, 3, 3).transpose(0, 2, 1)
    Vm = V.reshape(-1, 3, 3).transpose(0, 2, 1)
    Um = U.reshape(-1, 3, 3).transpose(0, 2, 1)
    # the reference factors A^T (svd3.h:1271-1274); its u*vt is V U^T of A
    np.testing.assert_allclose((Vm @ Um.transpose(0, 2, 1))[1:], R_ref[1:], atol=5e-5)
