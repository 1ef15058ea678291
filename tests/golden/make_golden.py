"""Generates tests/golden/*.npz from the reference's own arithmetic (oracle/_ref).

    python tests/golden/make_golden.py

Needs the reference sources (to build oracle/_ref/libcrmpm_ref.so).  Every fixture stores its
inputs next to the reference outputs, so tests/test_golden.py needs neither the reference nor the
scene builders' exact behaviour to check the CPU restatement against them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "cressim-mpm_b200"))

import oracle_py as op  # noqa: E402
from crmpm_b200 import scenes  # noqa: E402


def scene_arrays(sc):
    st = sc.shapes
    out = dict(solver_type=sc.solver_type, grid_min=sc.grid_min, grid_max=sc.grid_max, cell_size=sc.cell_size, dt=sc.dt,
               gravity=sc.gravity, iterations=sc.iterations, contact_model=sc.contact_model, pos_mass=sc.pos_mass,
               vel=sc.vel, mat_params=sc.mat_params, mat_type=sc.mat_type, mask=sc.mask)
    for k in ("shape_type", "geom_idx", "position", "rotation", "inv_scale", "lin_vel", "ang_vel", "com_inv_mass",
              "inertia0", "inertia1", "force", "torque", "params0", "geom_type", "geom_params", "sdf_dims", "sdf_lbcs",
              "sdf_data", "shape_ids"):
        out["sh_" + k] = getattr(st, k)
    return out


def run_case(name, sc, steps):
    r = op.RefOracle(sc)
    r.compute_initial_data()
    masks0 = r.cut_masks()
    st0 = r.state()
    r.step(steps)
    st = r.state()
    force, torque = r.coupling()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), steps=steps, **scene_arrays(sc),
                        V0_init=st0["V0"], masks0=masks0, x=st["x"], v=st["v"], F=st["F"], C=st["C"], V0=st["V0"],
                        force=force, torque=torque)
    print(name, sc.n, "particles,", steps, "steps")


def small_cube(**kw):
    return scenes.cube_drop(side=0.2, **kw)


def main():
    op.build(ref=True)
    assert op.ref_available(), "the reference driver could not be built"
    run_case("mls_cube", small_cube(), 100)
    run_case("mls_cube_linear", small_cube(material=scenes.MAT_LINEAR_ELASTIC), 60)
    run_case("std_cube", small_cube(solver=scenes.SOLVER_STANDARD, dt=1e-4), 60)
    pb = small_cube(solver=scenes.SOLVER_PB, dt=0.002)
    pb.mat_params[:, :2] = (1.0, 0.9)
    pb.iterations = 5
    run_case("pb_cube", pb, 10)
    for kind in ("quad_slicer", "mesh_slicer", "lines", "arc", "trimesh", "dynamic_sphere", "effmass_sphere",
                 "scaled_box", "capsule"):
        sc = scenes.contact_scene(kind)
        # keep fixtures small: every fourth particle
        for k in ("pos_mass", "vel", "mat_params", "mat_type", "mask"):
            setattr(sc, k, np.ascontiguousarray(getattr(sc, k)[::4]))
        run_case(f"contact_{kind}", sc, 40)

    # the SVD printout test of the reference (tests/test_svd/main.cpp:36) plus near-identity matrices
    rng = np.random.default_rng(7)
    A = np.vstack([np.array([[1, 2, 5, 3, 1, 4, 2, 9, 3]], np.float32),
                   (np.eye(3).ravel() + 0.1 * rng.normal(size=(63, 9))).astype(np.float32)])
    U, Vt, S = op.ref_svd3(A)
    np.savez_compressed(os.path.join(HERE, "svd3.npz"), A=A, U=U, Vt=Vt, S=S)

    # getGeometrySdf at random local points for every analytic and grid geometry
    out = {}
    for kind, gtype in (("box", scenes.GEOM_BOX), ("sphere", scenes.GEOM_SPHERE), ("plane", scenes.GEOM_PLANE),
                        ("capsule", scenes.GEOM_CAPSULE), ("arc", scenes.GEOM_ARC), ("lines", scenes.GEOM_CONNECTED_LINE_SEGMENTS),
                        ("trimesh", scenes.GEOM_TRIANGLE_MESH), ("quad_slicer", scenes.GEOM_QUAD_SLICER),
                        ("mesh_slicer", scenes.GEOM_TRIANGLE_MESH_SLICER)):
        sc = scenes.contact_scene(kind if kind not in ("box",) else "box")
        st = sc.shapes
        gid = int(st.geom_idx[st.shape_ids[0]])
        p0 = st.geom_params[gid]
        scale = 0.15 if kind != "arc" else 1.5
        pts = (rng.uniform(-1, 1, size=(256, 3)) * scale).astype(np.float32)
        res, tan, spine = op.sdf_query("ref", gtype, p0, st, pts)
        out[f"{kind}_gtype"] = gtype
        out[f"{kind}_params"] = p0
        out[f"{kind}_pts"] = pts
        out[f"{kind}_out"] = res
        out[f"{kind}_tan"] = tan
        out[f"{kind}_spine"] = spine
        for k in ("sdf_dims", "sdf_lbcs", "sdf_data"):
            out[f"{kind}_{k}"] = getattr(st, k)
    np.savez_compressed(os.path.join(HERE, "sdf_queries.npz"), **out)
    print("sdf queries and svd written")


if __name__ == "__main__":
    main()
