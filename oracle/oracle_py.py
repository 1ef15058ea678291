"""ORACLE / TEST INFRASTRUCTURE ONLY: ctypes bindings of the two CPU checkers.

* ``RefOracle``   drives oracle/_ref/libcrmpm_ref.so: the reference's own header-only substep
                  algorithms compiled for the host (oracle/ref_driver.cpp, oracle/Makefile).
* ``PortOracle``  drives oracle/liboracle.so: this repository's restatement of the same algorithms
                  (oracle/mpm_oracle.cpp), in float (reference operation order) or double.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libcrmpm_ref.so")
PORT_LIB = os.path.join(HERE, "liboracle.so")


class Float4P(C.c_void_p):
    pass


class ShapeDataC(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("type", "geometryIdx", "position", "rotation", "invScale",
                                          "linearVelocity", "angularVelocity", "comInvMass", "inertiaInv0",
                                          "inertiaInv1", "force", "torque", "params0")] + [("size", C.c_int)]


class GeometryDataC(C.Structure):
    _fields_ = [("type", C.c_void_p), ("params0", C.c_void_p), ("size", C.c_int)]


class GeometrySdfDataC(C.Structure):
    _fields_ = [("dimension", C.c_void_p), ("lowerBoundCellSize", C.c_void_p), ("gradientSignedDistance", C.c_void_p)]


def reference_root() -> str | None:
    """Where the reference's sources lie, as the oracle recipe (oracle/Makefile, `print-ref`) has
    it; None when that folder does not exist (on a machine that only runs the prebuilt oracle)."""
    try:
        r = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True, check=True)
    except (OSError, subprocess.CalledProcessError):
        return None
    path = r.stdout.strip()
    return path if path and os.path.isdir(path) else None


def build(ref: bool = True) -> None:
    """Compile the restatement (and, when the reference sources exist, the reference driver)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if ref and reference_root() is not None:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


class HostShapes:
    """Keeps contiguous host copies of a ShapeTable alive and exposes the three C structs."""

    def __init__(self, st):
        self.a = {}
        for k in ("shape_type", "geom_idx", "position", "rotation", "inv_scale", "lin_vel", "ang_vel",
                  "com_inv_mass", "inertia0", "inertia1", "force", "torque", "params0", "geom_type",
                  "geom_params", "sdf_dims", "sdf_lbcs", "sdf_data", "shape_ids"):
            v = getattr(st, k)
            if v.shape[0] == 0:
                v = np.zeros((1,) + v.shape[1:], v.dtype)
            self.a[k] = np.ascontiguousarray(v)
        a = self.a
        self.shapes = ShapeDataC(_p(a["shape_type"]), _p(a["geom_idx"]), _p(a["position"]), _p(a["rotation"]),
                                 _p(a["inv_scale"]), _p(a["lin_vel"]), _p(a["ang_vel"]), _p(a["com_inv_mass"]),
                                 _p(a["inertia0"]), _p(a["inertia1"]), _p(a["force"]), _p(a["torque"]),
                                 _p(a["params0"]), int(st.shape_type.shape[0]))
        self.geoms = GeometryDataC(_p(a["geom_type"]), _p(a["geom_params"]), int(st.geom_type.shape[0]))
        self.sdf = GeometrySdfDataC(_p(a["sdf_dims"]), _p(a["sdf_lbcs"]), _p(a["sdf_data"]))
        self.num = int(st.shape_ids.shape[0])


_ref_lib = None
_port_lib = None


def _load_ref():
    global _ref_lib
    if _ref_lib is None:
        lib = C.CDLL(REF_LIB)
        lib.ref_create.restype = C.c_void_p
        lib.ref_create.argtypes = [C.c_int, C.c_int, C.c_float, C.c_void_p, C.c_void_p]
        for fn in ("ref_destroy", "ref_step"):
            getattr(lib, fn).argtypes = [C.c_void_p]
        lib.ref_phase.argtypes = [C.c_void_p, C.c_int]
        lib.ref_grid_dims.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_set_params.argtypes = [C.c_void_p, C.c_float, C.c_void_p, C.c_int, C.c_int]
        lib.ref_bind_particles.argtypes = [C.c_void_p] + [C.c_void_p] * 5 + [C.c_uint]
        lib.ref_bind_shapes.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ref_compute_initial_data.argtypes = [C.c_void_p, C.c_uint, C.c_void_p]
        lib.ref_get_state.argtypes = [C.c_void_p, C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ref_set_state.argtypes = [C.c_void_p, C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ref_get_grid.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ref_set_grid.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_cut_masks.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_sdf_query.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p]
        lib.ref_svd3.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _ref_lib = lib
    return _ref_lib


def _load_port():
    global _port_lib
    if _port_lib is None:
        lib = C.CDLL(PORT_LIB)
        lib.orc_create.restype = C.c_void_p
        lib.orc_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p, C.c_void_p]
        for fn in ("orc_destroy", "orc_step", "orc_reset_coupling"):
            getattr(lib, fn).argtypes = [C.c_void_p]
        lib.orc_phase.argtypes = [C.c_void_p, C.c_int]
        lib.orc_grid_dims.argtypes = [C.c_void_p, C.c_void_p]
        lib.orc_set_params.argtypes = [C.c_void_p, C.c_float, C.c_void_p, C.c_int, C.c_int]
        lib.orc_set_state.argtypes = [C.c_void_p, C.c_uint] + [C.c_void_p] * 8 + [C.c_uint]
        lib.orc_get_state.argtypes = [C.c_void_p, C.c_uint] + [C.c_void_p] * 5
        lib.orc_bind_shapes.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.orc_get_coupling.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        lib.orc_compute_initial_data.argtypes = [C.c_void_p, C.c_uint, C.c_void_p]
        lib.orc_get_grid.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.orc_set_grid.argtypes = [C.c_void_p, C.c_void_p]
        lib.orc_cut_masks.argtypes = [C.c_void_p, C.c_void_p]
        lib.orc_sdf_query.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]
        lib.orc_svd3.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _port_lib = lib
    return _port_lib


class RefOracle:
    """The reference's own CPU arithmetic on one scene (float32 state, reference layouts)."""

    def __init__(self, scene, num_max: int | None = None):
        self.lib = _load_ref()
        self.scene = scene
        n = scene.n
        nmax = num_max or n
        self.nmax = nmax
        mn = np.ascontiguousarray(scene.grid_min, np.float32)
        mx = np.ascontiguousarray(scene.grid_max, np.float32)
        self.h = self.lib.ref_create(scene.solver_type, nmax, C.c_float(scene.cell_size), _p(mn), _p(mx))
        g = np.ascontiguousarray(scene.gravity, np.float32)
        self.lib.ref_set_params(self.h, C.c_float(scene.dt), _p(g), scene.iterations, scene.contact_model)

        def grow(a, fill=0):
            out = np.full((nmax,) + a.shape[1:], fill, a.dtype)
            out[:n] = a
            return np.ascontiguousarray(out)

        self.pos = grow(scene.pos_mass)
        self.vel = grow(scene.vel)
        self.matp = grow(scene.mat_params)
        self.matt = grow(scene.mat_type)
        self.mask = grow(scene.mask)
        self.lib.ref_bind_particles(self.h, _p(self.pos), _p(self.vel), _p(self.matp), _p(self.matt), _p(self.mask), n)
        self.hs = HostShapes(scene.shapes)
        self.lib.ref_bind_shapes(self.h, self.hs.num, _p(self.hs.a["shape_ids"]), C.byref(self.hs.shapes),
                                 C.byref(self.hs.geoms), C.byref(self.hs.sdf))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    def grid_dims(self):
        out = np.zeros(3, np.int32)
        self.lib.ref_grid_dims(self.h, _p(out))
        return tuple(int(v) for v in out)

    def compute_initial_data(self, idx=None):
        idx = np.arange(self.scene.n, dtype=np.uint32) if idx is None else np.ascontiguousarray(idx, np.uint32)
        self.lib.ref_compute_initial_data(self.h, idx.shape[0], _p(idx))

    def step(self, k: int = 1):
        for _ in range(k):
            self.lib.ref_step(self.h)

    def phase(self, p: int):
        self.lib.ref_phase(self.h, p)

    def state(self, n=None):
        n = self.scene.n if n is None else n
        F = np.zeros((n, 9), np.float32)
        Cm = np.zeros((n, 9), np.float32)
        V0 = np.zeros(n, np.float32)
        self.lib.ref_get_state(self.h, n, _p(F), _p(Cm), _p(V0))
        return dict(x=self.pos[:n, :3].copy(), m=self.pos[:n, 3].copy(), v=self.vel[:n, :3].copy(), F=F, C=Cm, V0=V0)

    def set_state(self, F=None, Cm=None, V0=None):
        n = self.scene.n
        a = [None if t is None else np.ascontiguousarray(t, np.float32) for t in (F, Cm, V0)]
        self.lib.ref_set_state(self.h, n, *[None if t is None else _p(t) for t in a])

    def grid(self):
        nx, ny, nz = self.grid_dims()
        g = np.zeros((nx * ny * nz, 4), np.float32)
        f = np.zeros((nx * ny * nz, 4), np.float32)
        self.lib.ref_get_grid(self.h, _p(g), _p(f))
        return g, f

    def set_grid(self, g):
        g = np.ascontiguousarray(g, np.float32)
        self.lib.ref_set_grid(self.h, _p(g))

    def cut_masks(self):
        out = np.zeros(self.scene.n, np.uint32)
        self.lib.ref_cut_masks(self.h, _p(out))
        return out

    def coupling(self):
        """Shape force/torque accumulated by the reference into the host shape arrays."""
        return self.hs.a["force"].copy(), self.hs.a["torque"].copy()


class PortOracle:
    """This repository's CPU restatement (prec 32 = reference order in float, 64 = FP64 oracle)."""

    def __init__(self, scene, prec: int = 64, num_max: int | None = None):
        self.lib = _load_port()
        self.scene = scene
        self.prec = prec
        n = scene.n
        self.nmax = num_max or n
        mn = np.ascontiguousarray(scene.grid_min, np.float32)
        mx = np.ascontiguousarray(scene.grid_max, np.float32)
        self.h = self.lib.orc_create(prec, scene.solver_type, self.nmax, C.c_float(scene.cell_size), _p(mn), _p(mx))
        g = np.ascontiguousarray(scene.gravity, np.float32)
        self.lib.orc_set_params(self.h, C.c_float(scene.dt), _p(g), scene.iterations, scene.contact_model)
        pm = np.ascontiguousarray(scene.pos_mass, np.float64)
        v = np.ascontiguousarray(scene.vel, np.float64)
        mp = np.ascontiguousarray(scene.mat_params, np.float64)
        mt = np.ascontiguousarray(scene.mat_type, np.int32)
        mk = np.ascontiguousarray(scene.mask, np.uint8)
        self.lib.orc_set_state(self.h, n, _p(pm), _p(v), None, None, None, _p(mp), _p(mt), _p(mk), n)
        self.hs = HostShapes(scene.shapes)
        self.lib.orc_bind_shapes(self.h, self.hs.num, _p(self.hs.a["shape_ids"]), C.byref(self.hs.shapes),
                                 C.byref(self.hs.geoms), C.byref(self.hs.sdf))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def grid_dims(self):
        out = np.zeros(3, np.int32)
        self.lib.orc_grid_dims(self.h, _p(out))
        return tuple(int(v) for v in out)

    def compute_initial_data(self, idx=None):
        idx = np.arange(self.scene.n, dtype=np.uint32) if idx is None else np.ascontiguousarray(idx, np.uint32)
        self.lib.orc_compute_initial_data(self.h, idx.shape[0], _p(idx))

    def step(self, k: int = 1):
        for _ in range(k):
            self.lib.orc_step(self.h)

    def phase(self, p: int):
        self.lib.orc_phase(self.h, p)

    def state(self, n=None):
        n = self.scene.n if n is None else n
        pm = np.zeros((n, 4))
        v = np.zeros((n, 4))
        F = np.zeros((n, 9))
        Cm = np.zeros((n, 9))
        V0 = np.zeros(n)
        self.lib.orc_get_state(self.h, n, _p(pm), _p(v), _p(F), _p(Cm), _p(V0))
        return dict(x=pm[:, :3], m=pm[:, 3], v=v[:, :3], F=F, C=Cm, V0=V0)

    def set_state(self, x=None, v=None, F=None, Cm=None, V0=None):
        n = self.scene.n
        pm = None
        if x is not None:
            pm = np.zeros((n, 4))
            pm[:, :3] = x
            pm[:, 3] = self.state(n)["m"]
        vv = None
        if v is not None:
            vv = np.zeros((n, 4))
            vv[:, :3] = v
        a = [None if t is None else np.ascontiguousarray(t, np.float64) for t in (pm, vv, F, Cm, V0)]
        self.lib.orc_set_state(self.h, n, *[None if t is None else _p(t) for t in a], None, None, None, n)

    def grid(self):
        nx, ny, nz = self.grid_dims()
        g = np.zeros((nx * ny * nz, 4))
        f = np.zeros((nx * ny * nz, 3))
        self.lib.orc_get_grid(self.h, _p(g), _p(f))
        return g, f

    def set_grid(self, g):
        g = np.ascontiguousarray(g, np.float64)
        self.lib.orc_set_grid(self.h, _p(g))

    def cut_masks(self):
        out = np.zeros(self.scene.n, np.uint32)
        self.lib.orc_cut_masks(self.h, _p(out))
        return out

    def coupling(self, shape_id: int):
        out = np.zeros(6)
        self.lib.orc_get_coupling(self.h, shape_id, _p(out))
        return out


def ref_svd3(A9: np.ndarray):
    lib = _load_ref()
    A = np.ascontiguousarray(A9, np.float32).reshape(-1, 9)
    n = A.shape[0]
    U = np.zeros((n, 9), np.float32)
    Vt = np.zeros((n, 9), np.float32)
    S = np.zeros((n, 3), np.float32)
    lib.ref_svd3(n, _p(A), _p(U), _p(Vt), _p(S))
    return U, Vt, S


def port_svd3(A9: np.ndarray, prec: int = 64):
    lib = _load_port()
    A = np.ascontiguousarray(A9, np.float64).reshape(-1, 9)
    n = A.shape[0]
    U = np.zeros((n, 9))
    V = np.zeros((n, 9))
    S = np.zeros((n, 3))
    lib.orc_svd3(prec, n, _p(A), _p(U), _p(V), _p(S))
    return U, V, S


def sdf_query(kind: str, geom_type: int, params0, st, pts: np.ndarray, prec: int = 32):
    """getGeometrySdf at local points with the reference ("ref") or the restatement ("port")."""
    hs = HostShapes(st)
    p0 = np.ascontiguousarray(params0, np.float32)
    n = pts.shape[0]
    if kind == "ref":
        lib = _load_ref()
        lp = np.zeros((n, 4), np.float32)
        lp[:, :3] = pts
        out = np.zeros((n, 4), np.float32)
        tan = np.zeros((n, 4), np.float32)
        sp = np.zeros(n, np.int32)
        lib.ref_sdf_query(geom_type, _p(p0), C.byref(hs.sdf), n, _p(lp), _p(out), _p(tan), _p(sp))
    else:
        lib = _load_port()
        lp = np.zeros((n, 4))
        lp[:, :3] = pts
        out = np.zeros((n, 4))
        tan = np.zeros((n, 4))
        sp = np.zeros(n, np.int32)
        lib.orc_sdf_query(prec, geom_type, _p(p0), C.byref(hs.sdf), n, _p(lp), _p(out), _p(tan), _p(sp))
    return out, tan, sp


# ---------------------------------------------------------------------------------------------
# Triangle-mesh SDF grids: the reference's own builder (oracle/_ref/libref_sdf.so) and the
# restatement (sdf_oracle.cpp in oracle/liboracle.so)
# ---------------------------------------------------------------------------------------------

REF_SDF_LIB = os.path.join(HERE, "_ref", "libref_sdf.so")
_ref_sdf_lib = None


def ref_sdf_available() -> bool:
    return os.path.exists(REF_SDF_LIB)


def _mesh(points, triangles):
    P = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    T = np.ascontiguousarray(triangles, np.uint32).reshape(-1, 3)
    return P, T


def _spine(spine):
    return np.asarray((np.nan, 0, 0, 0) if spine is None else spine, np.float32)


def ref_sdf(points, triangles, cell: float, fatten: float = 0.0, normalize: bool = True, slicer: bool = False,
            spine=None):
    """(dims, lower, grid [nx*ny*nz, 4]) from the reference's SdfBuilder run on the host."""
    global _ref_sdf_lib
    if _ref_sdf_lib is None:
        lib = C.CDLL(REF_SDF_LIB)
        lib.ref_sdf_desc.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_void_p,
                                     C.c_void_p]
        lib.ref_sdf_build.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_int,
                                      C.c_void_p]
        lib.ref_sdf_build_mod.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_float, C.c_float,
                                          C.c_void_p, C.c_void_p]
        _ref_sdf_lib = lib
    L = _ref_sdf_lib
    P, T = _mesh(points, triangles)
    dims = np.zeros(3, np.int32)
    lower = np.zeros(3, np.float32)
    L.ref_sdf_desc(_p(P), P.shape[0], _p(T), T.shape[0], cell, fatten, _p(dims), _p(lower))
    n = int(np.prod(dims.astype(np.int64)))
    out = np.zeros((n, 4), np.float32)
    if slicer:
        L.ref_sdf_build_mod(_p(P), P.shape[0], _p(T), T.shape[0], cell, fatten, _p(_spine(spine)), _p(out))
    else:
        L.ref_sdf_build(_p(P), P.shape[0], _p(T), T.shape[0], cell, fatten, int(normalize), _p(out))
    return tuple(int(v) for v in dims), lower, out


def port_sdf(points, triangles, cell: float, fatten: float = 0.0, normalize: bool = True, slicer: bool = False,
             spine=None):
    """(dims, lower, size, grid [nx*ny*nz, 4]) from the restatement (sdf_oracle.cpp)."""
    L = _load_port()
    if not getattr(L, "_sdf_sig", False):
        L.oracle_sdf_desc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_void_p, C.c_void_p,
                                      C.c_void_p]
        L.oracle_sdf_build.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_float,
                                       C.c_int, C.c_void_p, C.c_int, C.c_void_p]
        L._sdf_sig = True
    P, T = _mesh(points, triangles)
    dims = np.zeros(3, np.int32)
    lower = np.zeros(3, np.float32)
    size = np.zeros(3, np.float32)
    L.oracle_sdf_desc(_p(P), _p(T), T.shape[0], cell, fatten, _p(dims), _p(lower), _p(size))
    out = np.zeros((int(np.prod(dims.astype(np.int64))), 4), np.float32)
    sp = _spine(spine)
    L.oracle_sdf_build(_p(P), P.shape[0], _p(T), T.shape[0], _p(dims), _p(lower), cell, int(slicer), _p(sp),
                       int(normalize), _p(out))
    return tuple(int(v) for v in dims), lower, size, out


# The reference's own CUDA solvers (oracle/_ref/ref_gpu_driver, built by `make -C oracle ref-gpu`
# from src/solver/gpu_*_mpm_solver.cu): GPU-vs-GPU parity and the reference's GPU substep time.
REF_GPU_DRIVER = os.path.join(HERE, "_ref", "ref_gpu_driver")
_ANALYTIC_GEOMETRIES = (0, 1, 2, 3, 5, 8)  # box, sphere, plane, capsule, quad slicer, arc


def ref_gpu_available() -> bool:
    return os.path.exists(REF_GPU_DRIVER)


def write_ref_gpu_scene(sc, path: str) -> None:
    """Write a scene in the layout ref_gpu_driver.cu reads (analytic geometries only)."""
    st = sc.shapes
    if any(int(t) not in _ANALYTIC_GEOMETRIES for t in st.geom_type):
        raise ValueError("ref_gpu_driver takes analytic geometries only")
    f32 = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731
    i32 = lambda a: np.ascontiguousarray(a, np.int32)  # noqa: E731
    with open(path, "wb") as f:
        i32([sc.n, sc.solver_type, sc.iterations, sc.contact_model]).tofile(f)
        f32([sc.cell_size, sc.dt, *sc.grid_min, *sc.grid_max, *sc.gravity]).tofile(f)
        for a in (sc.pos_mass, sc.vel, sc.mat_params):
            f32(a).tofile(f)
        i32(sc.mat_type).tofile(f)
        np.ascontiguousarray(sc.mask, np.uint8).tofile(f)
        S = int(st.shape_type.shape[0])
        i32([S]).tofile(f)
        i32(st.shape_type).tofile(f)
        i32(st.geom_idx).tofile(f)
        for a in (st.position, st.rotation, st.inv_scale, st.lin_vel, st.ang_vel, st.com_inv_mass, st.inertia0,
                  st.inertia1, st.params0):
            f32(a).reshape(S, 4).tofile(f)
        i32([st.shape_ids.shape[0]]).tofile(f)
        i32(st.shape_ids).tofile(f)
        i32([st.geom_type.shape[0]]).tofile(f)
        i32(st.geom_type).tofile(f)
        f32(st.geom_params).tofile(f)
        i32([st.sdf_dims.shape[0]]).tofile(f)
        i32(st.sdf_dims).tofile(f)
        f32(st.sdf_lbcs).tofile(f)
        i32([st.sdf_data.shape[0]]).tofile(f)
        f32(st.sdf_data).tofile(f)


def ref_gpu_run(sc, steps: int, warmup: int = 0, workdir: str = None, timeout: float = 600.0) -> dict:
    """Run the reference's CUDA solver on `sc`: `warmup` substeps, then `steps` timed ones.

    Returns {"x", "v" [n,3], "force", "torque" [S,4], "ms_per_substep"}; the state is after
    warmup + steps substeps.
    """
    import tempfile

    with tempfile.TemporaryDirectory(dir=workdir) as d:
        scene, out = os.path.join(d, "scene.bin"), os.path.join(d, "out.bin")
        write_ref_gpu_scene(sc, scene)
        r = subprocess.run([REF_GPU_DRIVER, scene, str(warmup), str(steps), out], capture_output=True, text=True,
                           timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_gpu_driver exited {r.returncode}: {r.stdout}{r.stderr}")
        S = int(sc.shapes.shape_type.shape[0])
        res = np.fromfile(out, np.float32)
    n = sc.n
    pm, vel = res[:4 * n].reshape(n, 4), res[4 * n:8 * n].reshape(n, 4)
    ft = res[8 * n:].reshape(2, S, 4)
    ms = float(r.stdout.split()[1])
    return {"x": pm[:, :3].copy(), "mass": pm[:, 3].copy(), "v": vel[:, :3].copy(), "force": ft[0], "torque": ft[1],
            "ms_per_substep": ms}
