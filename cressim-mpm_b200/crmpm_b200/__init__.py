"""Python mirror of the B200 MPM engine's C ABI (include/crmpm_b200.h).

``GpuSolver`` exposes the reference solver interface (``MpmSolver``,
include/solver/mpm_solver.h:63-191) method for method: ``initialize``, ``step``,
``fetch_results``, ``compute_initial_data``, the setters and the ``bind_*`` calls take device
pointers exactly like the reference's GPU solvers.  ``DeviceScene`` owns the device buffers of one
scene (as the reference's ``SceneImpl`` does, src/engine/scene_impl.cpp:42-93) and is what tests
and the benchmark drive.

The compute path is libcrmpm_b200.so only: importing this module fails loudly if the library is
missing, and nothing here falls back to a CPU implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import scenes  # noqa: F401  (re-exported for convenience)

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "libcrmpm_b200.so")
ROOT = os.path.dirname(PKG)
HEADER = os.path.join(ROOT, "include", "crmpm_b200.h")

OK = 0
ERR_TIMEOUT = -7
STATUS_NAN_STATE = 0x1
STATUS_BLOCK_OVERFLOW = 0x2
STATUS_OUT_OF_DOMAIN = 0x4
OPT_PHASE_TIMING = 3
OPT_DETERMINISTIC_COUPLING = 4
OPT_DETERMINISTIC = 5
OPT_RESIDENT = 6
OPT_STANDARD_GPU_SEMANTICS = 7
PHASES = ("sort", "p2g", "grid_update", "g2p")


class CrmpmError(RuntimeError):
    pass


class ShapeDataC(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("type", "geometryIdx", "position", "rotation", "invScale",
                                          "linearVelocity", "angularVelocity", "comInvMass", "inertiaInv0",
                                          "inertiaInv1", "force", "torque", "params0")] + [("size", C.c_int)]


class GeometryDataC(C.Structure):
    _fields_ = [("type", C.c_void_p), ("params0", C.c_void_p), ("size", C.c_int)]


class GeometrySdfDataC(C.Structure):
    _fields_ = [("dimension", C.c_void_p), ("lowerBoundCellSize", C.c_void_p), ("gradientSignedDistance", C.c_void_p)]


class NoAllocStepC(C.Structure):
    """CrB200NoAllocStep (include/crmpm_b200.h)."""

    _fields_ = [("gridMin", C.c_float * 3), ("gridMax", C.c_float * 3), ("cellSize", C.c_float), ("dt", C.c_float),
                ("gravity", C.c_float * 3), ("contactModel", C.c_int), ("numParticles", C.c_uint),
                ("positionMass", C.c_void_p), ("velocity", C.c_void_p), ("F", C.c_void_p), ("C", C.c_void_p),
                ("V0", C.c_void_p), ("matParams", C.c_void_p), ("matType", C.c_void_p), ("activeMask", C.c_void_p),
                ("numShapes", C.c_int), ("shapeIds", C.c_void_p), ("shapes", ShapeDataC),
                ("geometries", GeometryDataC), ("sdf", GeometrySdfDataC)]


class BatchSceneDescC(C.Structure):
    """CrB200BatchSceneDesc (include/crmpm_b200.h)."""

    _fields_ = [("gridMin", C.c_float * 3), ("gridMax", C.c_float * 3), ("cellSize", C.c_float), ("dt", C.c_float),
                ("gravity", C.c_float * 3), ("contactModel", C.c_int), ("particleOffset", C.c_uint),
                ("numParticles", C.c_uint), ("shapeOffset", C.c_int), ("numShapes", C.c_int)]


class TriangleMeshC(C.Structure):
    """CrB200TriangleMesh (include/crmpm_b200.h)."""

    _fields_ = [("points", C.c_void_p), ("triangles", C.c_void_p), ("numPoints", C.c_int), ("numTriangles", C.c_int)]


class SdfDescC(C.Structure):
    """CrB200SdfDesc (include/crmpm_b200.h)."""

    _fields_ = [("cellSize", C.c_float), ("fatten", C.c_float), ("slicerSpineArea", C.c_float * 4),
                ("boundingSize", C.c_float * 3), ("lowerBound", C.c_float * 3), ("sdfDimension", C.c_int * 3)]


_lib = None


def build_library(force: bool = False) -> str:
    """Compile libcrmpm_b200.so in place (nvcc, sm_100a)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("crmpm_b200_build", os.path.join(PKG, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(force=force)


def lib() -> C.CDLL:
    """The loaded C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CrmpmError(f"{LIB_PATH} is missing: build it with `python cressim-mpm_b200/build.py`")
    L = C.CDLL(LIB_PATH)
    vp, i, u, f = C.c_void_p, C.c_int, C.c_uint, C.c_float
    sig = {
        "CrB200GetLastError": (C.c_char_p, []),
        "CrB200GetVersion": (i, []),
        "CrB200GetKernelLaunchCount": (C.c_uint64, []),
        "CrB200SolverCreate": (i, [i, i, f, vp, vp, vp, C.POINTER(vp)]),
        "CrB200SolverRelease": (i, [vp]),
        "CrB200SolverInitialize": (i, [vp]),
        "CrB200SolverStep": (i, [vp, C.POINTER(f)]),
        "CrB200SolverStepMany": (i, [vp, i]),
        "CrB200SolverFetchResults": (i, [vp]),
        "CrB200SolverComputeInitialData": (i, [vp, u, vp]),
        "CrB200SolverSetGravity": (i, [vp, f, f, f]),
        "CrB200SolverSetIntegrationStepSize": (i, [vp, f]),
        "CrB200SolverSetSolverIterations": (i, [vp, i]),
        "CrB200SolverSetShapeContactModel": (i, [vp, i]),
        "CrB200SolverSetNumActiveParticles": (i, [vp, u]),
        "CrB200SolverBindParticleData": (i, [vp, vp, vp]),
        "CrB200SolverBindParticleMaterials": (i, [vp, vp, vp]),
        "CrB200SolverBindActiveMask": (i, [vp, vp]),
        "CrB200SolverSetNumShapes": (i, [vp, i]),
        "CrB200SolverBindShapeIds": (i, [vp, vp]),
        "CrB200SolverBindShapeData": (i, [vp, vp]),
        "CrB200SolverBindGeometryData": (i, [vp, vp]),
        "CrB200SolverBindGeometrySdfData": (i, [vp, vp]),
        "CrB200SolverGetGridDims": (i, [vp, vp]),
        "CrB200SolverCopyParticleState": (i, [vp, u, vp, vp, vp]),
        "CrB200SolverSetParticleState": (i, [vp, u, vp, vp, vp]),
        "CrB200SolverCopySortState": (i, [vp, vp, vp, C.POINTER(u)]),
        "CrB200SolverCopyCutMasks": (i, [vp, vp]),
        "CrB200SolverGetStatus": (i, [vp, C.POINTER(u), i]),
        "CrB200SolverClearStatus": (i, [vp]),
        "CrB200SolverSetOption": (i, [vp, i, i]),
        "CrB200SolverAdvance": (i, [vp, f, vp, vp, C.POINTER(i)]),
        "CrB200SolverAdvanceAsync": (i, [vp, f, vp, vp, C.POINTER(i)]),
        "CrB200SolverGetPhaseTimes": (i, [vp, vp, C.POINTER(i), i]),
        "CrB200SolverGetGridStats": (i, [vp, vp]),
        "CrB200SolverGetResidentKernelTime": (i, [vp, C.POINTER(f), C.POINTER(i), i]),
        "CrB200SolverGetFp64Fallbacks": (i, [vp, C.POINTER(u), i]),
        "CrB200SvdBatch": (i, [u, vp, vp, vp, vp, vp, vp, vp, vp]),
        "CrB200MlsSubstepNoAlloc": (i, [C.POINTER(NoAllocStepC), vp]),
        "CrB200BatchCreate": (i, [i, i, vp, i, i, vp, C.POINTER(vp)]),
        "CrB200SolverAdjointRecord": (i, [vp, i, i, i, vp, vp]),
        "CrB200SolverAutotune": (i, [vp, i, vp]),
        "CrB200SolverAdjointBackward": (i, [vp, vp, vp, vp, vp]),
        "CrB200SdfPrecomputeDesc": (i, [C.POINTER(SdfDescC), C.POINTER(TriangleMeshC)]),
        "CrB200SdfCompute": (i, [C.POINTER(SdfDescC), C.POINTER(TriangleMeshC), vp, i, vp]),
        "CrB200SdfComputeMod": (i, [C.POINTER(SdfDescC), C.POINTER(TriangleMeshC), vp, vp]),
        "CrB200SdfGetLastKernelTime": (i, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def declared_symbols() -> list[str]:
    """Every function name declared in include/crmpm_b200.h."""
    import re

    txt = open(HEADER).read()
    return sorted(set(re.findall(r"CRB200_API\s+[\w\s\*]+?\b(CrB200\w+)\s*\(", txt)))


def check(rc: int, what: str = "") -> None:
    if rc != OK:
        msg = lib().CrB200GetLastError().decode()
        raise CrmpmError(f"{what} failed ({rc}): {msg}")


def kernel_launch_count() -> int:
    return int(lib().CrB200GetKernelLaunchCount())


class SdfGrid:
    """An SDF grid built on the GPU: ``data`` is a torch float32 tensor [nz, ny, nx, 4] on the device
    (gradient xyz, distance w; the flat layout the solvers' gradientSignedDistance arrays hold),
    ``dims`` (nx, ny, nz), ``lower`` the position of node (0, 0, 0), ``cell`` the node spacing."""

    def __init__(self, data, dims, lower, cell, size):
        self.data, self.dims, self.lower, self.cell, self.size = data, dims, lower, cell, size

    def host(self) -> np.ndarray:
        """Flat float32 [nx * ny * nz, 4] copy in node order (x fastest)."""
        return self.data.reshape(-1, 4).cpu().numpy()


def _mesh_struct(points: np.ndarray, triangles: np.ndarray):
    P = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    T = np.ascontiguousarray(triangles, np.uint32).reshape(-1, 3)
    m = TriangleMeshC(P.ctypes.data, T.ctypes.data, P.shape[0], T.shape[0])
    return m, (P, T)


def sdf_desc(points, triangles, cell_size: float, fatten: float = 0.0, spine=None) -> SdfDescC:
    """SdfBuilder::precomputeSdfDesc (src/geometry_utils/sdf_builder.cpp:84-103) via
    CrB200SdfPrecomputeDesc: the grid the reference lays over the mesh."""
    m, keep = _mesh_struct(points, triangles)
    d = SdfDescC()
    d.cellSize = float(cell_size)
    d.fatten = float(fatten)
    sp = (float("nan"), 0.0, 0.0, 0.0) if spine is None else tuple(float(v) for v in spine)
    d.slicerSpineArea = (C.c_float * 4)(*sp)
    check(lib().CrB200SdfPrecomputeDesc(C.byref(d), C.byref(m)), "CrB200SdfPrecomputeDesc")
    del keep
    return d


def build_sdf(points, triangles, cell_size: float, fatten: float = 0.0, normalize: bool = True,
              slicer: bool = False, spine=None, device=None, out=None, stream: int | None = None) -> SdfGrid:
    """Build the SDF grid of a triangle mesh on the GPU, as the reference's factory does when it
    creates an eTriangleMesh geometry (computeSdf + computeSdfGradient) or, with ``slicer``, an
    eTriangleMeshSlicer geometry (computeModSdf + computeSdfGradient + postProcessModSdfGradient,
    spine plane ``spine`` = (nx, ny, nz, d) or None).  ``out``: optional device tensor of
    nx * ny * nz * 4 float32 to write into (e.g. a slice of a scene's SDF data array)."""
    import torch

    d = sdf_desc(points, triangles, cell_size, fatten, spine)
    nx, ny, nz = (int(v) for v in d.sdfDimension)
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if out is None:
        out = torch.empty((nz, ny, nx, 4), dtype=torch.float32, device=dev)
    elif out.numel() != nx * ny * nz * 4 or out.dtype != torch.float32 or not out.is_contiguous():
        raise CrmpmError("build_sdf: `out` must be a contiguous float32 tensor of nx * ny * nz * 4 elements")
    m, keep = _mesh_struct(points, triangles)
    st = C.c_void_p(stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream)
    if slicer:
        check(lib().CrB200SdfComputeMod(C.byref(d), C.byref(m), C.c_void_p(out.data_ptr()), st), "CrB200SdfComputeMod")
    else:
        check(lib().CrB200SdfCompute(C.byref(d), C.byref(m), C.c_void_p(out.data_ptr()), int(bool(normalize)), st),
              "CrB200SdfCompute")
    del keep
    return SdfGrid(out, (nx, ny, nz), tuple(float(v) for v in d.lowerBound), float(d.cellSize),
                   tuple(float(v) for v in d.boundingSize))


def sdf_last_kernel_ms() -> tuple[float, float]:
    """GPU times (distance kernel, gradient kernel) in ms of the last build_sdf on this thread
    (CrB200SdfGetLastKernelTime)."""
    ms = (C.c_float * 2)()
    check(lib().CrB200SdfGetLastKernelTime(ms), "CrB200SdfGetLastKernelTime")
    return float(ms[0]), float(ms[1])


class GpuSolver:
    """One B200 solver behind the reference's MpmSolver interface (device pointers are ints)."""

    def __init__(self, solver_type: int, num_max_particles: int, cell_size: float, grid_min, grid_max,
                 stream: int | None = None):
        L = lib()
        mn = (C.c_float * 3)(*[float(v) for v in grid_min])
        mx = (C.c_float * 3)(*[float(v) for v in grid_max])
        h = C.c_void_p()
        check(L.CrB200SolverCreate(int(solver_type), int(num_max_particles), C.c_float(cell_size), mn, mx,
                                   C.c_void_p(stream or 0), C.byref(h)), "CrB200SolverCreate")
        self._h = h
        self._keep = []

    @classmethod
    def batch(cls, solver_type: int, descs, num_max_particles: int, iterations: int,
              stream: int | None = None) -> "GpuSolver":
        """A solver over many scenes (CrB200BatchCreate); ``descs`` is a list of BatchSceneDescC."""
        arr = (BatchSceneDescC * len(descs))(*descs)
        h = C.c_void_p()
        check(lib().CrB200BatchCreate(int(solver_type), len(descs), arr, int(num_max_particles), int(iterations),
                                      C.c_void_p(stream or 0), C.byref(h)), "CrB200BatchCreate")
        self = cls.__new__(cls)
        self._h = h
        self._keep = [arr]
        return self

    def release(self) -> None:
        if self._h:
            check(lib().CrB200SolverRelease(self._h), "release")
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    # -- MpmSolver -------------------------------------------------------------------------
    def initialize(self):
        check(lib().CrB200SolverInitialize(self._h), "initialize")

    def step(self) -> float:
        dt = C.c_float()
        check(lib().CrB200SolverStep(self._h, C.byref(dt)), "step")
        return dt.value

    def step_many(self, n: int):
        check(lib().CrB200SolverStepMany(self._h, int(n)), "step_many")

    def fetch_results(self):
        check(lib().CrB200SolverFetchResults(self._h), "fetch_results")

    def compute_initial_data(self, n: int, indices_ptr: int):
        check(lib().CrB200SolverComputeInitialData(self._h, int(n), C.c_void_p(indices_ptr)), "compute_initial_data")

    def set_gravity(self, g):
        check(lib().CrB200SolverSetGravity(self._h, *[C.c_float(float(v)) for v in g]), "set_gravity")

    def set_integration_step_size(self, dt: float):
        check(lib().CrB200SolverSetIntegrationStepSize(self._h, C.c_float(dt)), "set_integration_step_size")

    def set_solver_iterations(self, n: int):
        check(lib().CrB200SolverSetSolverIterations(self._h, int(n)), "set_solver_iterations")

    def set_shape_contact_model(self, m: int):
        check(lib().CrB200SolverSetShapeContactModel(self._h, int(m)), "set_shape_contact_model")

    def set_num_active_particles(self, n: int):
        check(lib().CrB200SolverSetNumActiveParticles(self._h, int(n)), "set_num_active_particles")

    def bind_particle_data(self, pos_ptr: int, vel_ptr: int):
        check(lib().CrB200SolverBindParticleData(self._h, C.c_void_p(pos_ptr), C.c_void_p(vel_ptr)), "bind_particle_data")

    def bind_particle_materials(self, params_ptr: int, type_ptr: int):
        check(lib().CrB200SolverBindParticleMaterials(self._h, C.c_void_p(params_ptr), C.c_void_p(type_ptr)),
              "bind_particle_materials")

    def bind_active_mask(self, mask_ptr: int):
        check(lib().CrB200SolverBindActiveMask(self._h, C.c_void_p(mask_ptr)), "bind_active_mask")

    def set_num_shapes(self, n: int):
        check(lib().CrB200SolverSetNumShapes(self._h, int(n)), "set_num_shapes")

    def bind_shape_ids(self, ptr: int):
        check(lib().CrB200SolverBindShapeIds(self._h, C.c_void_p(ptr)), "bind_shape_ids")

    def bind_shape_data(self, sd: ShapeDataC):
        self._keep.append(sd)
        check(lib().CrB200SolverBindShapeData(self._h, C.byref(sd)), "bind_shape_data")

    def bind_geometry_data(self, gd: GeometryDataC):
        self._keep.append(gd)
        check(lib().CrB200SolverBindGeometryData(self._h, C.byref(gd)), "bind_geometry_data")

    def bind_geometry_sdf_data(self, sd: GeometrySdfDataC):
        self._keep.append(sd)
        check(lib().CrB200SolverBindGeometrySdfData(self._h, C.byref(sd)), "bind_geometry_sdf_data")

    # -- additions ---------------------------------------------------------------------------
    def grid_dims(self):
        out = (C.c_int * 3)()
        check(lib().CrB200SolverGetGridDims(self._h, out), "grid_dims")
        return tuple(out)

    def copy_particle_state(self, n: int, F_ptr=0, C_ptr=0, V0_ptr=0):
        check(lib().CrB200SolverCopyParticleState(self._h, int(n), C.c_void_p(F_ptr), C.c_void_p(C_ptr),
                                                  C.c_void_p(V0_ptr)), "copy_particle_state")

    def set_particle_state(self, n: int, F_ptr=0, C_ptr=0, V0_ptr=0):
        check(lib().CrB200SolverSetParticleState(self._h, int(n), C.c_void_p(F_ptr), C.c_void_p(C_ptr),
                                                 C.c_void_p(V0_ptr)), "set_particle_state")

    def copy_sort_state(self, keys_ptr=0, ids_ptr=0) -> int:
        n = C.c_uint()
        check(lib().CrB200SolverCopySortState(self._h, C.c_void_p(keys_ptr), C.c_void_p(ids_ptr), C.byref(n)),
              "copy_sort_state")
        return n.value

    def copy_cut_masks(self, ptr: int):
        check(lib().CrB200SolverCopyCutMasks(self._h, C.c_void_p(ptr)), "copy_cut_masks")

    def status(self, timeout_ms: int = 1000) -> int:
        s = C.c_uint()
        check(lib().CrB200SolverGetStatus(self._h, C.byref(s), int(timeout_ms)), "status")
        return s.value

    def clear_status(self):
        check(lib().CrB200SolverClearStatus(self._h), "clear_status")

    def set_option(self, opt: int, value: int):
        check(lib().CrB200SolverSetOption(self._h, int(opt), int(value)), "set_option")

    def advance(self, dt: float, host_pos_ptr: int = 0, host_vel_ptr: int = 0) -> int:
        """Scene-style advance: substeps until the float time reaches dt, then read back x / v."""
        n = C.c_int()
        check(lib().CrB200SolverAdvance(self._h, C.c_float(dt), C.c_void_p(host_pos_ptr), C.c_void_p(host_vel_ptr),
                                        C.byref(n)), "advance")
        return n.value

    def advance_async(self, dt: float, host_pos_ptr: int = 0, host_vel_ptr: int = 0) -> int:
        """advance without waiting: the readback into the host buffers completes by fetch_results()."""
        n = C.c_int()
        check(lib().CrB200SolverAdvanceAsync(self._h, C.c_float(dt), C.c_void_p(host_pos_ptr),
                                             C.c_void_p(host_vel_ptr), C.byref(n)), "advance_async")
        return n.value

    def phase_times(self, reset: bool = True):
        ms = (C.c_float * 4)()
        n = C.c_int()
        check(lib().CrB200SolverGetPhaseTimes(self._h, ms, C.byref(n), int(reset)), "phase_times")
        return list(ms), n.value

    def fp64_fallbacks(self, reset: bool = False) -> int:
        """PB-MPM SVDs redone in double precision since the last reset."""
        out = C.c_uint()
        check(lib().CrB200SolverGetFp64Fallbacks(self._h, C.byref(out), int(reset)), "fp64_fallbacks")
        return out.value

    def resident_kernel_time(self, reset: bool = True):
        """(milliseconds, launches) of the resident path's fused G2P -> P2G kernel under phase timing."""
        ms = C.c_float()
        n = C.c_int()
        check(lib().CrB200SolverGetResidentKernelTime(self._h, C.byref(ms), C.byref(n), int(reset)),
              "resident_kernel_time")
        return ms.value, n.value

    def autotune(self, substeps_per_trial: int = 8):
        """Pick the fastest launch shapes (CrB200SolverAutotune); returns (update CTAs per SM,
        accumulation multiple, sort multiple)."""
        out = (C.c_int * 3)()
        check(lib().CrB200SolverAutotune(self._h, int(substeps_per_trial), out), "autotune")
        return tuple(out)

    def adjoint_record(self, num_substeps: int, interval: int, captures, captured_ptr: int):
        caps = (C.c_int * max(len(captures), 1))(*[int(t) for t in captures])
        check(lib().CrB200SolverAdjointRecord(self._h, int(num_substeps), int(interval), len(captures), caps,
                                              C.c_void_p(captured_ptr)), "adjoint_record")

    def adjoint_backward(self, grad_ptr: int, grad_v_ptr: int = 0, grad_mat_ptr: int = 0, grad_x_ptr: int = 0):
        check(lib().CrB200SolverAdjointBackward(self._h, C.c_void_p(grad_ptr), C.c_void_p(grad_v_ptr),
                                                C.c_void_p(grad_mat_ptr), C.c_void_p(grad_x_ptr)), "adjoint_backward")

    def grid_stats(self):
        out = (C.c_uint * 4)()
        check(lib().CrB200SolverGetGridStats(self._h, out), "grid_stats")
        return dict(num_sorted=out[0], active_blocks=out[1], touched_blocks=out[2], touched_nodes=out[3])


def svd_batch(A9, device: str = "cuda:0"):
    """The engine's device SVD (CrB200SvdBatch) of column-major 3x3 matrices [n, 9]: U, V [n, 9],
    S [n, 3], the PB-MPM rotation target R [n, 9], fp64-redo flags [n] and their count."""
    import torch

    A = torch.as_tensor(np.ascontiguousarray(A9, np.float32).reshape(-1, 9), device=device)
    n = A.shape[0]
    U, V, R = (torch.empty((n, 9), dtype=torch.float32, device=device) for _ in range(3))
    S = torch.empty((n, 3), dtype=torch.float32, device=device)
    used = torch.empty(max(n, 1), dtype=torch.int32, device=device)
    count = torch.zeros(1, dtype=torch.int32, device=device)
    stream = torch.cuda.current_stream(device)
    check(lib().CrB200SvdBatch(n, A.data_ptr(), U.data_ptr(), V.data_ptr(), S.data_ptr(), R.data_ptr(),
                               used.data_ptr(), count.data_ptr(), C.c_void_p(stream.cuda_stream)), "svd_batch")
    torch.cuda.synchronize(device)
    return (U.cpu().numpy(), V.cpu().numpy(), S.cpu().numpy(), R.cpu().numpy(), used[:n].cpu().numpy(),
            int(count.item()))


class DeviceScene:
    """Device buffers of one scene bound to a GpuSolver (torch is used for device memory only)."""

    def __init__(self, scene, num_max: int | None = None, device: str = "cuda:0", stream=None,
                 compute_initial: bool = True):
        import torch

        self.torch = torch
        self.scene = scene
        self.device = torch.device(device)
        n = scene.n
        self.num_max = num_max or n
        self.stream = stream if stream is not None else torch.cuda.Stream(device=self.device)
        dev = self.device

        def up(a, dtype=None, rows=None):
            a = np.ascontiguousarray(a)
            if rows is not None and a.shape[0] < rows:
                pad = np.zeros((rows - a.shape[0],) + a.shape[1:], a.dtype)
                a = np.concatenate([a, pad])
            t = torch.from_numpy(a).to(dev)
            return t

        nm = self.num_max
        self.pos = up(scene.pos_mass, rows=nm)
        self.vel = up(scene.vel, rows=nm)
        self.matp = up(scene.mat_params, rows=nm)
        self.matt = up(scene.mat_type.astype(np.int32), rows=nm)
        self.mask = up(scene.mask.astype(np.uint8), rows=nm)
        st = scene.shapes
        self.sh = {}
        for k in ("shape_type", "geom_idx", "position", "rotation", "inv_scale", "lin_vel", "ang_vel", "com_inv_mass",
                  "inertia0", "inertia1", "force", "torque", "params0", "geom_type", "geom_params", "sdf_dims",
                  "sdf_lbcs", "sdf_data", "shape_ids"):
            v = getattr(st, k)
            if v.shape[0] == 0:
                v = np.zeros((1,) + v.shape[1:], v.dtype)
            self.sh[k] = up(v)
        torch.cuda.synchronize(dev)
        self.solver = self._create_solver(scene, nm)
        s = self.solver
        s.bind_particle_data(self.pos.data_ptr(), self.vel.data_ptr())
        s.bind_particle_materials(self.matp.data_ptr(), self.matt.data_ptr())
        s.bind_active_mask(self.mask.data_ptr())
        p = {k: v.data_ptr() for k, v in self.sh.items()}
        s.bind_shape_data(ShapeDataC(p["shape_type"], p["geom_idx"], p["position"], p["rotation"], p["inv_scale"],
                                     p["lin_vel"], p["ang_vel"], p["com_inv_mass"], p["inertia0"], p["inertia1"],
                                     p["force"], p["torque"], p["params0"], int(st.shape_type.shape[0])))
        s.bind_geometry_data(GeometryDataC(p["geom_type"], p["geom_params"], int(st.geom_type.shape[0])))
        s.bind_geometry_sdf_data(GeometrySdfDataC(p["sdf_dims"], p["sdf_lbcs"], p["sdf_data"]))
        s.bind_shape_ids(p["shape_ids"])
        self._set_counts(s, scene)
        s.initialize()
        if compute_initial:
            self.compute_initial_data()

    def _create_solver(self, scene, nm: int) -> GpuSolver:
        s = GpuSolver(scene.solver_type, nm, scene.cell_size, scene.grid_min, scene.grid_max,
                      stream=self.stream.cuda_stream)
        s.set_gravity(scene.gravity)
        s.set_integration_step_size(scene.dt)
        s.set_solver_iterations(scene.iterations)
        s.set_shape_contact_model(scene.contact_model)
        return s

    def _set_counts(self, s: GpuSolver, scene) -> None:
        s.set_num_active_particles(scene.n)
        s.set_num_shapes(scene.shapes.num_shapes)

    def compute_initial_data(self, idx=None):
        torch = self.torch
        idx = np.arange(self.scene.n, dtype=np.uint32) if idx is None else np.asarray(idx, np.uint32)
        self._idx = torch.from_numpy(idx.astype(np.int32)).to(self.device)
        torch.cuda.synchronize(self.device)
        self.solver.compute_initial_data(idx.shape[0], self._idx.data_ptr())

    def step(self, k: int = 1, graph: bool = True):
        if graph and k > 1:
            self.solver.step_many(k)
        else:
            for _ in range(k):
                self.solver.step()

    def sync(self):
        self.solver.fetch_results()

    def set_shape(self, shape_id: int, position=None, lin_vel=None, rotation=None, ang_vel=None):
        """Update one shape's pose / velocity on the solver stream (what a factory sync does)."""
        torch = self.torch
        with torch.cuda.stream(self.stream):
            for key, val in (("position", position), ("lin_vel", lin_vel), ("rotation", rotation), ("ang_vel", ang_vel)):
                if val is not None:
                    v = list(val) + [0.0] * (4 - len(val))
                    self.sh[key][shape_id] = torch.tensor(v[:4], dtype=torch.float32, device=self.device)

    def state(self):
        torch = self.torch
        n = self.scene.n
        F = torch.empty((n, 9), dtype=torch.float32, device=self.device)
        Cm = torch.empty((n, 9), dtype=torch.float32, device=self.device)
        V0 = torch.empty(n, dtype=torch.float32, device=self.device)
        self.solver.copy_particle_state(n, F.data_ptr(), Cm.data_ptr(), V0.data_ptr())
        self.sync()
        return dict(x=self.pos[:n, :3].cpu().numpy(), m=self.pos[:n, 3].cpu().numpy(), v=self.vel[:n, :3].cpu().numpy(),
                    F=F.cpu().numpy(), C=Cm.cpu().numpy(), V0=V0.cpu().numpy())

    def set_state(self, F=None, Cm=None, V0=None):
        torch = self.torch
        n = self.scene.n
        ts = [None if a is None else torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(self.device)
              for a in (F, Cm, V0)]
        torch.cuda.synchronize(self.device)
        self.solver.set_particle_state(n, *[0 if t is None else t.data_ptr() for t in ts])
        self.sync()

    def sort_state(self):
        torch = self.torch
        n = self.scene.n
        keys = torch.empty(max(n, 1), dtype=torch.int32, device=self.device)
        ids = torch.empty(max(n, 1), dtype=torch.int32, device=self.device)
        cnt = self.solver.copy_sort_state(keys.data_ptr(), ids.data_ptr())
        self.sync()
        return keys[:n].cpu().numpy().view(np.uint32), ids[:cnt].cpu().numpy().view(np.uint32)

    def cut_masks(self):
        torch = self.torch
        n = self.scene.n
        out = torch.empty(max(n, 1), dtype=torch.int32, device=self.device)
        self.solver.copy_cut_masks(out.data_ptr())
        self.sync()
        return out[:n].cpu().numpy().view(np.uint32)

    def coupling(self):
        self.sync()
        return self.sh["force"].cpu().numpy(), self.sh["torque"].cpu().numpy()


class DeviceBatch(DeviceScene):
    """Many independent scenes advanced by one batch solver (CrB200BatchCreate).

    Particles of all scenes share one set of device arrays (scene s at ``batch.slice(s)``) and
    their shapes one merged shape table; ``state()`` returns the concatenated arrays and
    ``scene_state(s)`` one scene's part.
    """

    def __init__(self, scene_list, device: str = "cuda:0", stream=None, compute_initial: bool = True):
        from . import scenes as _scenes

        self.batch = _scenes.make_batch(scene_list)
        super().__init__(self.batch.merged, device=device, stream=stream, compute_initial=compute_initial)

    def _create_solver(self, scene, nm: int) -> GpuSolver:
        b = self.batch
        descs = []
        for k, sc in enumerate(b.scenes):
            d = BatchSceneDescC()
            d.gridMin[:] = [float(v) for v in sc.grid_min]
            d.gridMax[:] = [float(v) for v in sc.grid_max]
            d.cellSize = float(sc.cell_size)
            d.dt = float(sc.dt)
            d.gravity[:] = [float(v) for v in sc.gravity]
            d.contactModel = int(sc.contact_model)
            d.particleOffset = int(b.particle_offset[k])
            d.numParticles = int(sc.n)
            d.shapeOffset = int(b.shape_offset[k])
            d.numShapes = int(sc.shapes.num_shapes)
            descs.append(d)
        return GpuSolver.batch(scene.solver_type, descs, nm, scene.iterations, stream=self.stream.cuda_stream)

    def _set_counts(self, s: GpuSolver, scene) -> None:
        pass  # the descriptors carry every scene's particle and shape ranges

    def scene_state(self, s: int, state: dict | None = None) -> dict:
        st = self.state() if state is None else state
        sl = self.batch.slice(s)
        return {k: v[sl] for k, v in st.items()}
