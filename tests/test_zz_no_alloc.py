"""The allocation-free MLS substep (CrB200MlsSubstepNoAlloc) against the regular solver.

Some callers cannot call cudaMalloc where they step the simulation -- a host that has already
split all device memory among its own pools, or a real-time loop that must not block on an
allocation.  For them the library offers one substep entry point whose only scratch is a fixed
static device array.  This file checks, through the C ABI, that two calls in a row give the same
particle state as two substeps of the regular solver (CrB200SolverStep) within the tolerances of
the other parity tests, and that oversized grids are refused.  It is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from conftest import cuda_available
from gpu_helpers import rel_pos_err

import crmpm_b200 as cb
from crmpm_b200 import scenes


def _desc(sc, t, stream_shapes):
    d = cb.NoAllocStepC()
    d.gridMin = (ctypes.c_float * 3)(*[float(v) for v in sc.grid_min])
    d.gridMax = (ctypes.c_float * 3)(*[float(v) for v in sc.grid_max])
    d.cellSize = sc.cell_size
    d.dt = sc.dt
    d.gravity = (ctypes.c_float * 3)(*[float(v) for v in sc.gravity])
    d.contactModel = sc.contact_model
    d.numParticles = sc.n
    for name in ("positionMass", "velocity", "F", "C", "V0", "matParams", "matType", "activeMask"):
        setattr(d, name, t[name].data_ptr() if t.get(name) is not None else None)
    sh = stream_shapes
    d.numShapes = sc.shapes.num_shapes
    d.shapeIds = sh["shape_ids"].data_ptr()
    d.shapes = cb.ShapeDataC(*[sh[k].data_ptr() for k in ("shape_type", "geom_idx", "position", "rotation", "inv_scale",
                                                          "lin_vel", "ang_vel", "com_inv_mass", "inertia0", "inertia1",
                                                          "force", "torque", "params0")],
                             int(sc.shapes.shape_type.shape[0]))
    d.geometries = cb.GeometryDataC(sh["geom_type"].data_ptr(), sh["geom_params"].data_ptr(),
                                    int(sc.shapes.geom_type.shape[0]))
    d.sdf = cb.GeometrySdfDataC(sh["sdf_dims"].data_ptr(), sh["sdf_lbcs"].data_ptr(), sh["sdf_data"].data_ptr())
    return d


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")
@pytest.mark.parametrize("kind", ["cube", "quad_slicer", "effmass_sphere", "dynamic_sphere"])
def test_no_alloc_substep_matches_solver_step(kind):
    """Two calls in a row against two CrB200SolverStep substeps of the same scene: particle state
    within the parity tolerances, and for the dynamic-shape scenes (the effective-mass contact
    model and the kinematic one) the coupling force and torque the grid contact accumulates on the
    shape.  After the two calls the particle positions are also checked against the FP64 oracle
    directly, so the entry point is pinned independently of the regular solver."""
    import torch

    import oracle_py as op

    cb.build_library()
    sc = scenes.cube_drop() if kind == "cube" else scenes.contact_scene(kind)
    ref = cb.DeviceScene(sc)  # the existing entry points (allocating solver)
    st0 = ref.state()
    dev = ref.device
    t = {
        "positionMass": torch.from_numpy(sc.pos_mass.copy()).to(dev),
        "velocity": torch.from_numpy(sc.vel.copy()).to(dev),
        "F": torch.from_numpy(st0["F"].copy()).to(dev),
        "C": torch.from_numpy(st0["C"].copy()).to(dev),
        "V0": torch.from_numpy(st0["V0"].copy()).to(dev),
        "matParams": ref.matp[: sc.n].clone(),
        "matType": ref.matt[: sc.n].clone(),
        "activeMask": ref.mask[: sc.n].clone(),
    }
    shapes = {k: v.clone() for k, v in ref.sh.items()}
    d = _desc(sc, t, shapes)
    stream = torch.cuda.current_stream(dev)
    L = cb.lib()
    torch.cuda.synchronize(dev)
    for call in range(2):
        ref.step(1, graph=False)
        rc = L.CrB200MlsSubstepNoAlloc(ctypes.byref(d), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.CrB200GetLastError().decode()
        torch.cuda.synchronize(dev)
        a = ref.state()
        x = t["positionMass"][:, :3].cpu().numpy()
        v = t["velocity"][:, :3].cpu().numpy()
        F = t["F"].cpu().numpy()
        Cm = t["C"].cpu().numpy()
        assert rel_pos_err(x, a["x"], sc.pos_mass[:, :3], sc.cell_size) <= 1e-4, f"call {call}"
        vscale = max(float(np.abs(a["v"]).max()), 1e-3)
        assert float(np.abs(v - a["v"]).max()) <= 1e-3 * vscale, f"call {call}"
        assert float(np.abs(F - a["F"]).max()) <= 1e-4, f"call {call}"
        cscale = max(float(np.abs(a["C"]).max()), 1e-3)
        assert float(np.abs(Cm - a["C"]).max()) <= 1e-3 * cscale, f"call {call}"
        if kind.endswith("_sphere"):
            # the dynamic shape's coupling force and torque, accumulated over the calls so far
            f_ref, q_ref = ref.coupling()
            for name, got, exp in (("force", shapes["force"], f_ref), ("torque", shapes["torque"], q_ref)):
                got = got.cpu().numpy()[:, :3]
                exp = exp[:, :3]
                scale = max(float(np.abs(exp).max()), 1e-6)
                assert float(np.abs(got - exp).max()) <= 1e-3 * scale, f"{name}, call {call}"
    o = op.PortOracle(sc, 64)
    o.compute_initial_data()
    o.step(2)
    x64 = o.state()["x"]
    x = t["positionMass"][:, :3].cpu().numpy()
    assert rel_pos_err(x, x64, sc.pos_mass[:, :3], sc.cell_size) <= 1e-4


def test_no_alloc_rejects_oversized_grid():
    L = cb.lib()
    d = cb.NoAllocStepC()
    d.gridMin = (ctypes.c_float * 3)(-1, -1, -1)
    d.gridMax = (ctypes.c_float * 3)(1, 1, 1)
    d.cellSize = 0.02  # 101^3 nodes > 262,144
    d.dt = 1e-4
    d.numParticles = 0
    d.numShapes = 0
    rc = L.CrB200MlsSubstepNoAlloc(ctypes.byref(d), None)
    assert rc == -6
    assert b"262144" in L.CrB200GetLastError()
