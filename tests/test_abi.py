"""C-ABI checks that need no GPU: the library loads and exports every declared entry point."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import crmpm_b200 as cb


def test_library_builds_and_loads():
    cb.build_library()
    assert os.path.exists(cb.LIB_PATH)
    L = cb.lib()
    assert L.CrB200GetVersion() == 100


def test_every_declared_symbol_is_exported():
    declared = cb.declared_symbols()
    assert len(declared) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", cb.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    # nothing beyond the declared C ABI leaks out of the library
    extra = sorted(s for s in exported if s.startswith("CrB200") and s not in declared)
    assert not extra, extra


def test_create_rejects_bad_arguments_without_gpu():
    L = cb.lib()
    h = ctypes.c_void_p()
    mn = (ctypes.c_float * 3)(0, 0, 0)
    mx = (ctypes.c_float * 3)(1, 1, 1)
    # CPU solver kinds have no counterpart here
    assert L.CrB200SolverCreate(0, 10, ctypes.c_float(0.1), mn, mx, None, ctypes.byref(h)) == -3
    assert b"GPU solver types" in L.CrB200GetLastError()
    assert L.CrB200SolverCreate(1, 0, ctypes.c_float(0.1), mn, mx, None, ctypes.byref(h)) == -1
    assert L.CrB200SolverCreate(1, 10, ctypes.c_float(-1.0), mn, mx, None, ctypes.byref(h)) == -1
    assert L.CrB200SolverCreate(1, 10, ctypes.c_float(0.5), mn, mx, None, ctypes.byref(h)) == -1  # < 5 nodes
    assert L.CrB200SolverRelease(None) == -1


def test_grid_dims_match_reference_formula():
    from crmpm_b200 import scenes

    L = cb.lib()
    for sc in (scenes.cube_drop(), scenes.tissue_slab(size=(0.2, 0.1, 0.2)), scenes.pb_cutting(size=(0.1, 0.05, 0.1))):
        s = cb.GpuSolver(sc.solver_type, 16, sc.cell_size, sc.grid_min, sc.grid_max)
        assert s.grid_dims() == sc.grid_dims()
        s.release()


def _desc(off, n, soff=0, ns=0, mn=(-1, -1, -1), mx=(1, 1, 1), cell=0.1):
    d = cb.BatchSceneDescC()
    d.gridMin[:] = mn
    d.gridMax[:] = mx
    d.cellSize, d.dt = cell, 1e-4
    d.gravity[:] = (0, -9.81, 0)
    d.contactModel = 0
    d.particleOffset, d.numParticles, d.shapeOffset, d.numShapes = off, n, soff, ns
    return d


def test_batch_desc_layout():
    # 11 floats, 1 int, 2 unsigned, 2 int: the C struct has no padding
    assert ctypes.sizeof(cb.BatchSceneDescC) == 64


def test_batch_create_validates_scenes_without_gpu():
    L = cb.lib()

    def create(descs, nmax=1000, solver=1):
        arr = (cb.BatchSceneDescC * len(descs))(*descs)
        h = ctypes.c_void_p()
        rc = L.CrB200BatchCreate(solver, len(descs), arr, nmax, 10, None, ctypes.byref(h))
        if rc == 0:
            assert L.CrB200SolverRelease(h) == 0
        return rc

    assert create([_desc(0, 100), _desc(100, 200, 1, 2)]) == 0
    assert create([_desc(0, 100), _desc(50, 100)]) == -1  # overlapping particle ranges
    assert b"overlap" in L.CrB200GetLastError()
    assert create([_desc(0, 100), _desc(900, 200)]) == -6  # past numMaxParticles
    assert create([_desc(0, 10, 0, 65)]) == -6  # more than 64 shapes in one scene
    assert create([_desc(0, 10, cell=0.6)]) == -1  # fewer than 5 nodes per dimension
    assert create([_desc(0, 10)], solver=2) == -3
    assert create([]) == -1


def test_batch_refuses_single_scene_counts():
    s = cb.GpuSolver.batch(1, [_desc(0, 10), _desc(10, 10)], 100, 10)
    with pytest.raises(cb.CrmpmError):
        s.set_num_active_particles(5)
    with pytest.raises(cb.CrmpmError):
        s.set_num_shapes(1)
    s.release()


def test_merge_shape_tables_shifts_sdf_references():
    from crmpm_b200 import scenes

    a, b = scenes.contact_scene("trimesh"), scenes.contact_scene("mesh_slicer")
    merged, offs = scenes.merge_shape_tables([a.shapes, b.shapes])
    assert offs == [0, a.shapes.num_shapes]
    assert merged.shape_ids.shape[0] == a.shapes.num_shapes + b.shapes.num_shapes
    ga = a.shapes.geom_type.shape[0]
    for gi, gt in enumerate(b.shapes.geom_type):
        if int(gt) in scenes._SDF_GEOMS:
            off, sid = b.shapes.geom_params[gi, :2].view(np.int32)
            moff, msid = merged.geom_params[ga + gi, :2].view(np.int32)
            assert moff == off + a.shapes.sdf_data.shape[0] and msid == sid + a.shapes.sdf_dims.shape[0]
            # the merged table holds the same SDF block at the shifted place
            np.testing.assert_array_equal(merged.sdf_dims[msid], b.shapes.sdf_dims[sid])
            np.testing.assert_array_equal(merged.sdf_data[moff], b.shapes.sdf_data[off])
