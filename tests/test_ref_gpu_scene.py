"""The scene file that oracle/_ref/ref_gpu_driver reads (the reference's CUDA solvers as a checker):
its byte layout, and the refusal of SDF-backed geometries, whose offsets the driver does not
check.  Host only."""
import numpy as np
import pytest

import oracle_py as op
from crmpm_b200 import scenes


def _expected_bytes(sc):
    st = sc.shapes
    S, K = st.shape_type.shape[0], st.shape_ids.shape[0]
    G, D, M = st.geom_type.shape[0], st.sdf_dims.shape[0], st.sdf_data.shape[0]
    return (16 + 44 + sc.n * (3 * 16 + 4 + 1) + 4 + S * (8 + 9 * 16) + 4 + 4 * K + 4 + G * (4 + 16) + 4 + D * 32
            + 4 + M * 16)


@pytest.mark.parametrize("make", [scenes.cube_drop, lambda: scenes.tissue_slab(size=(0.2, 0.1, 0.2)),
                                  lambda: scenes.pb_cutting(size=(0.1, 0.05, 0.1))])
def test_scene_file_layout(make, tmp_path):
    sc = make()
    path = tmp_path / "scene.bin"
    op.write_ref_gpu_scene(sc, str(path))
    raw = path.read_bytes()
    assert len(raw) == _expected_bytes(sc)
    hdr = np.frombuffer(raw[:16], np.int32)
    assert list(hdr) == [sc.n, sc.solver_type, sc.iterations, sc.contact_model]
    f = np.frombuffer(raw[16:60], np.float32)
    np.testing.assert_array_equal(f[:2], np.float32([sc.cell_size, sc.dt]))
    np.testing.assert_array_equal(f[2:5], sc.grid_min)
    np.testing.assert_array_equal(f[5:8], sc.grid_max)
    pm = np.frombuffer(raw[60:60 + 16 * sc.n], np.float32).reshape(sc.n, 4)
    np.testing.assert_array_equal(pm, sc.pos_mass)


def test_scene_file_refuses_sdf_geometry(tmp_path):
    sc, _ = scenes.mesh_contact_scene((9, 9, 9), (-0.2, -0.2, -0.2), 0.05)
    assert any(int(t) in (4, 6, 7) for t in sc.shapes.geom_type)
    with pytest.raises(ValueError, match="analytic"):
        op.write_ref_gpu_scene(sc, str(tmp_path / "scene.bin"))
