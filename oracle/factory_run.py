"""ORACLE / TEST INFRASTRUCTURE ONLY: runs a scene through the reference's own C API
(c_api/include/crmpm_c_api.h:127-280) in one of the factory builds of build_factory.sh and writes
the particle state after the last frame, the shapes' coupling force and torque, and the wall time
of every frame (CrAdvance + CrFetchResults, the scene's own readback included).

Each build exports the same C symbols, so every run is its own process:

    python oracle/factory_run.py LIB SCENE FRAMES OUT.npz [SPARE] [--cpu]

SCENE: cube_mls, cube_pb, cube_standard (a 0.1 m Neo-Hookean cube dropped on a ground plane) or
slab (the 1.0 x 0.2 x 1.0 m tissue slab, dx 0.01, particle spacing 0.005: about 1.6M particles,
the four side faces held by static boxes, a kinematic sphere probe moving down at 0.1 m/s).
Particles come from the reference's own particle-object sampler (a lattice inside the geometry,
particle_object_impl.cpp:36-86).  SPARE (default 1.0): numMaxParticles of the scene as a multiple of
the particles the object adds, to show what a scene's readback of numMaxParticles costs.  --cpu:
the factory builds no GPU data, so every scene falls back to the reference's CPU solvers
(simulation_factory_impl.cpp:351-378); it runs without a GPU.
"""
import ctypes as C
import sys
import time

import numpy as np


class Vec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class Vec4(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float), ("w", C.c_float)]


class Bounds3(C.Structure):
    _fields_ = [("center", Vec3), ("extents", Vec3)]


class ParticleData(C.Structure):
    _fields_ = [("numParticles", C.c_uint), ("positionMass", C.c_void_p), ("velocity", C.c_void_p)]


# enums of the reference (include/solver/mpm_solver.h:51-61, include/engine/shape.h:48-53,
# include/engine/geometry.h:41-60, include/solver/material_data.h:40-45)
SOLVER = {"cube_mls": 1, "cube_pb": 3, "cube_standard": 5, "slab": 1}
SHAPE_STATIC, SHAPE_KINEMATIC = 0, 1
GEOM_BOX, GEOM_SPHERE, GEOM_PLANE = 0, 1, 2
MAT_NEOHOOKEAN = 1


def _bind(lib):
    H = C.c_void_p
    sig = {
        "CrInitializeEngine": (None, [C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_int, C.c_int]),
        "CrGetInitializationStatus": (C.c_int, []),
        "CrReleaseEngine": (None, []),
        "CrAdvance": (None, [H, C.c_float]),
        "CrFetchResults": (None, [H]),
        "CrGetParticleData": (ParticleData, [H]),
        "CrGetShapeCouplingForceTorque": (None, [H, C.POINTER(Vec4), C.POINTER(Vec4)]),
        "CrCreateScene": (H, [C.c_int, C.c_int, Vec3, Bounds3, C.c_float, C.c_float, C.c_int, C.c_int]),
        "CrCreateShape": (H, [H, Vec3, Vec4, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, Vec3, Vec4, Vec4,
                              Vec4]),
        "CrCreateGeometry": (H, [C.c_int, Vec4]),
        "CrCreateParticleObject": (H, [C.c_float, C.c_float, H, C.POINTER(Vec3), C.POINTER(Vec4), C.POINTER(Vec3),
                                       C.c_int, C.POINTER(Vec4), C.POINTER(C.c_uint)]),
        "CrAddParticleObjectToScene": (None, [H, H, C.POINTER(C.c_uint)]),
        "CrAddShapeToScene": (None, [H, H]),
        "CrSetShapeVelocity": (None, [H, C.POINTER(Vec3), C.POINTER(Vec3)]),
        "CrReleaseScene": (None, [H]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def _lame(E, nu):
    return E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), E / (2.0 * (1.0 + nu))


def _bounds(lo, hi):
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    c, e = (lo + hi) / 2, (hi - lo) / 2
    return Bounds3(Vec3(*c), Vec3(*e))


def build(lib, scene, spare):
    """The scene through the C API: (scene handle, shape handles, particles added, numMaxParticles, substep)."""
    ident, one, zero4 = Vec4(0, 0, 0, 1), Vec3(1, 1, 1), Vec4(0, 0, 0, 0)
    shapes = []
    if scene.startswith("cube"):
        spacing, rho, cell, dt = 0.005, 1000.0, 0.01, 2e-4
        lam, mu = _lame(1e4, 0.3)
        mp = Vec4(lam, mu, 0, 0) if scene != "cube_pb" else Vec4(1.0, 0.9, 0, 0)
        geo = lib.CrCreateGeometry(GEOM_BOX, Vec4(0.05, 0.05, 0.05, 0))
        # 5.7 mm above the ground (contact after about 34 ms), off the grid planes by a fraction
        # of a spacing
        pos = Vec3(0.0013, 0.0557, -0.0021)
        bounds = _bounds((-0.3, -0.1, -0.3), (0.3, 0.4, 0.3))
    else:
        spacing, rho, cell, dt = 0.005, 1050.0, 0.01, 1e-4
        lam, mu = _lame(2e4, 0.4)
        mp = Vec4(lam, mu, 0, 0)
        geo = lib.CrCreateGeometry(GEOM_BOX, Vec4(0.5, 0.1, 0.5, 0))
        pos = Vec3(0.0013, 0.1007, -0.0021)
        bounds = _bounds((-0.6, -0.1, -0.6), (0.6, 0.5, 0.6))
    iterations = 10
    n = C.c_uint(0)
    rot = Vec4(0, 0, 0, 1)
    obj = lib.CrCreateParticleObject(spacing, rho * spacing ** 3, geo, C.byref(pos), C.byref(rot), C.byref(one),
                                     MAT_NEOHOOKEAN, C.byref(mp), C.byref(n))
    nmax = int(n.value * max(spare, 1.0))
    # Gravity leans a little (0.3 degrees) so that no grid node next to a shape moves exactly
    # parallel to its face: the reference applies contact only to nodes that approach a shape
    # (mpm_rigid_contact.h:187-191), and on a particle lattice at rest the tangential node
    # velocities would otherwise be rounding noise whose sign decides it (and friction with them).
    g = Vec3(0.05, -9.81, 0.03)
    sc = lib.CrCreateScene(SOLVER[scene], nmax, g, bounds, cell, dt, iterations, 0)
    off = C.c_uint(0)
    lib.CrAddParticleObjectToScene(obj, sc, C.byref(off))
    if scene.startswith("cube"):
        gp = lib.CrCreateGeometry(GEOM_PLANE, Vec4(0, 0, 0, 0))
        shapes.append(lib.CrCreateShape(gp, Vec3(0, 0, 0), ident, SHAPE_STATIC, 0.0, 0.0, 1.0, 0.3, one, zero4,
                                        zero4, zero4))
    else:
        # The pins abut the slab's faces and move with its offset, so that the edges of their
        # contact bands (one cell from the faces) lie off the planes of grid nodes.  On a node
        # plane the band test compares a distance that rounds to either side of the band width,
        # and the reference's CUDA build (contracted multiply-adds) and its CPU build round it
        # differently.
        t, sx, sy, sz = 0.02, 1.0, 0.2, 1.0
        o = (pos.x, pos.y - sy / 2, pos.z)
        gx = lib.CrCreateGeometry(GEOM_BOX, Vec4(t, sy / 2 + t, sz / 2 + 2 * t, 0))
        gz = lib.CrCreateGeometry(GEOM_BOX, Vec4(sx / 2 + 2 * t, sy / 2 + t, t, 0))
        for sgn in (-1.0, 1.0):
            shapes.append(lib.CrCreateShape(gx, Vec3(o[0] + sgn * (sx / 2 + t), o[1] + sy / 2, o[2]), ident,
                                            SHAPE_STATIC, cell, 0.0, 0.0, 0.0, one, zero4, zero4, zero4))
            shapes.append(lib.CrCreateShape(gz, Vec3(o[0], o[1] + sy / 2, o[2] + sgn * (sz / 2 + t)), ident,
                                            SHAPE_STATIC, cell, 0.0, 0.0, 0.0, one, zero4, zero4, zero4))
        gs = lib.CrCreateGeometry(GEOM_SPHERE, Vec4(0.05, 0, 0, 0))
        shapes.append(lib.CrCreateShape(gs, Vec3(o[0], o[1] + sy + 0.05 + cell, o[2]), ident, SHAPE_KINEMATIC, 0.0,
                                        0.0, 1.0, 0.3, one, zero4, zero4, zero4))
    for s in shapes:
        lib.CrAddShapeToScene(s, sc)
    if scene == "slab":
        lib.CrSetShapeVelocity(shapes[-1], C.byref(Vec3(0, -0.1, 0)), C.byref(Vec3(0, 0, 0)))
    return sc, shapes, int(n.value), nmax, dt


def main():
    args = [a for a in sys.argv[1:] if a != "--cpu"]
    gpu = "--cpu" not in sys.argv[1:]
    path, scene, frames, out = args[0], args[1], int(args[2]), args[3]
    spare = float(args[4]) if len(args) > 4 else 1.0
    lib = _bind(C.CDLL(path))
    substeps = 10
    probe_n = 2_000_000 if scene == "slab" else 200_000
    lib.CrInitializeEngine(int(probe_n * max(spare, 1.0)) + 1024, 64, 64, 1024, 1 if gpu else 0, 1)
    if lib.CrGetInitializationStatus() == 0:
        raise SystemExit("CrInitializeEngine failed")
    sc, shapes, n, nmax, dt = build(lib, scene, spare)
    frame_dt = substeps * dt
    # the substeps SceneImpl runs per frame: `while (t < dt) t += step()` in float
    # (scene_impl.cpp:313-317), which can run one more than frame_dt / dt
    t, per_frame = np.float32(0.0), 0
    while t < np.float32(frame_dt):
        t = np.float32(t + np.float32(dt))
        per_frame += 1

    def particles(pd, count):
        x = np.ctypeslib.as_array(C.cast(pd.positionMass, C.POINTER(C.c_float)), shape=(count, 4)).copy()
        v = np.ctypeslib.as_array(C.cast(pd.velocity, C.POINTER(C.c_float)), shape=(count, 4)).copy()
        return x, v

    pd0 = lib.CrGetParticleData(sc)
    x0, _ = particles(pd0, n)
    times = []
    for _ in range(frames):
        t0 = time.perf_counter()
        lib.CrAdvance(sc, frame_dt)
        lib.CrFetchResults(sc)
        times.append(time.perf_counter() - t0)
    pd = lib.CrGetParticleData(sc)
    assert pd.numParticles == n
    x, v = particles(pd, n)
    f, tq = Vec4(), Vec4()
    ft = []
    for s in shapes:
        lib.CrGetShapeCouplingForceTorque(s, C.byref(f), C.byref(tq))
        ft.append([f.x, f.y, f.z, tq.x, tq.y, tq.z])
    np.savez(out, x0=x0, x=x, v=v, times=np.array(times), n=n, nmax=nmax, coupling=np.array(ft, np.float64),
             substeps=per_frame)
    lib.CrReleaseScene(sc)
    lib.CrReleaseEngine()
    print(f"{scene} n={n} nmax={nmax} frames={frames} substeps per frame {per_frame} "
          f"median frame {np.median(times) * 1e3:.3f} ms")


if __name__ == "__main__":
    main()
