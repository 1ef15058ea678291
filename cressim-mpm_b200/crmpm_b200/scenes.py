"""Seeded synthetic scenes for the MPM substep engine.

Every scene is plain numpy data laid out like the reference's struct-of-arrays inputs:
particle position/mass and velocity as float4 (``ParticleData``, include/solver/particle_data.h:44-56),
material params0/type (``ParticleMaterialData``, include/solver/material_data.h:44-62), and the
rigid-shape / geometry / SDF tables (``ShapeData`` include/engine/shape.h:58-89, ``GeometryData``
include/engine/geometry.h:65-108, ``GeometrySdfData`` include/engine/geometry.h:113-118).

Particles are placed ``ppc`` per grid cell by seeded uniform jitter inside each cell.  The jitter
of particle ``k`` is drawn from SplitMix64 keyed by (seed, 3k + component), so a scene is a pure
function of its parameters.  Particle ids run cell by cell with x fastest, which keeps neighbouring
ids spatially close, the same ordering the reference's lattice sampler produces
(src/engine/particle_object_impl.cpp:52-82).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

SOLVER_MLS = 1
SOLVER_PB = 3
SOLVER_STANDARD = 5

MAT_COROTATIONAL = 0
MAT_NEOHOOKEAN = 1
MAT_LINEAR_ELASTIC = 2

SHAPE_STATIC = 0
SHAPE_KINEMATIC = 1
SHAPE_DYNAMIC = 2

GEOM_BOX = 0
GEOM_SPHERE = 1
GEOM_PLANE = 2
GEOM_CAPSULE = 3
GEOM_TRIANGLE_MESH = 4
GEOM_QUAD_SLICER = 5
GEOM_TRIANGLE_MESH_SLICER = 6
GEOM_CONNECTED_LINE_SEGMENTS = 7
GEOM_ARC = 8

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser on uint64 arrays (Steele, Lea, Flood 2014)."""
    with np.errstate(over="ignore"):
        z = (x.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)) & _M64
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, counters: np.ndarray) -> np.ndarray:
    """float32 in [0, 1) with 24 random bits from SplitMix64(seed << 32 | counter)."""
    key = (np.uint64(seed) << np.uint64(32)) + counters.astype(np.uint64)
    bits = splitmix64(key) >> np.uint64(40)
    return (bits.astype(np.float64) / float(1 << 24)).astype(np.float32)


def lame(E: float, nu: float) -> tuple[float, float]:
    """Lame parameters as the reference's tests compute them (tests/test_benchmark/main.cu:111-114)."""
    lam = (E * nu) / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    return float(np.float32(lam)), float(np.float32(mu))


def jittered_box(lo, hi, cell: float, ppc: int, seed: int, index_base: int = 0) -> np.ndarray:
    """Positions (float32 [N,3]) of ``ppc`` jittered particles per cell of the box [lo, hi]."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    counts = np.maximum(np.rint((hi - lo) / cell).astype(np.int64), 1)
    cz, cy, cx = np.meshgrid(np.arange(counts[2]), np.arange(counts[1]), np.arange(counts[0]), indexing="ij")
    corner = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1).astype(np.float64) * cell + lo
    corner = np.repeat(corner, ppc, axis=0)
    n = corner.shape[0]
    ctr = (np.arange(n, dtype=np.uint64) + np.uint64(index_base)) * np.uint64(3)
    jit = np.stack([uniform01(seed, ctr + np.uint64(c)) for c in range(3)], axis=1).astype(np.float64)
    return (corner + jit * cell).astype(np.float32)


@dataclasses.dataclass
class ShapeTable:
    """Host struct-of-arrays mirror of ShapeData / GeometryData / GeometrySdfData."""

    shape_type: np.ndarray  # int32 [S]
    geom_idx: np.ndarray  # int32 [S]
    position: np.ndarray  # float32 [S,4]
    rotation: np.ndarray  # float32 [S,4] quaternion x, y, z, w
    inv_scale: np.ndarray  # float32 [S,4]
    lin_vel: np.ndarray  # float32 [S,4]
    ang_vel: np.ndarray  # float32 [S,4]
    com_inv_mass: np.ndarray  # float32 [S,4]
    inertia0: np.ndarray  # float32 [S,4]
    inertia1: np.ndarray  # float32 [S,4]
    force: np.ndarray  # float32 [S,4]
    torque: np.ndarray  # float32 [S,4]
    params0: np.ndarray  # float32 [S,4] smooth, drag, friction, fatten
    geom_type: np.ndarray  # int32 [G]
    geom_params: np.ndarray  # float32 [G,4]
    sdf_dims: np.ndarray  # int32 [D,4]
    sdf_lbcs: np.ndarray  # float32 [D,4]
    sdf_data: np.ndarray  # float32 [M,4]
    shape_ids: np.ndarray  # int32 [numShapes in the scene]

    @staticmethod
    def empty() -> "ShapeTable":
        z4 = np.zeros((0, 4), np.float32)
        return ShapeTable(np.zeros(0, np.int32), np.zeros(0, np.int32), *(z4.copy() for _ in range(11)),
                          np.zeros(0, np.int32), z4.copy(), np.zeros((1, 4), np.int32),
                          np.zeros((1, 4), np.float32), np.zeros((1, 4), np.float32), np.zeros(0, np.int32))

    @property
    def num_shapes(self) -> int:
        return int(self.shape_ids.shape[0])

    def add_geometry(self, gtype: int, params) -> int:
        self.geom_type = np.append(self.geom_type, np.int32(gtype)).astype(np.int32)
        self.geom_params = np.vstack([self.geom_params, np.asarray(params, np.float32).reshape(1, 4)])
        return self.geom_type.shape[0] - 1

    def add_shape(self, geom: int, stype: int, position, rotation=(0, 0, 0, 1), inv_scale=(1, 1, 1),
                  smooth: float = 0.0, drag: float = 1.0, friction: float = 0.0, fatten: float = 0.0,
                  lin_vel=(0, 0, 0), ang_vel=(0, 0, 0), com_inv_mass=(0, 0, 0, 0), inertia0=(0, 0, 0, 0),
                  inertia1=(0, 0, 0, 0), in_scene: bool = True) -> int:
        def f4(v):
            v = list(v) + [0.0] * (4 - len(v))
            return np.asarray(v[:4], np.float32).reshape(1, 4)

        self.shape_type = np.append(self.shape_type, np.int32(stype)).astype(np.int32)
        self.geom_idx = np.append(self.geom_idx, np.int32(geom)).astype(np.int32)
        self.position = np.vstack([self.position, f4(position)])
        self.rotation = np.vstack([self.rotation, np.asarray(rotation, np.float32).reshape(1, 4)])
        self.inv_scale = np.vstack([self.inv_scale, f4(inv_scale)])
        self.lin_vel = np.vstack([self.lin_vel, f4(lin_vel)])
        self.ang_vel = np.vstack([self.ang_vel, f4(ang_vel)])
        self.com_inv_mass = np.vstack([self.com_inv_mass, f4(com_inv_mass)])
        self.inertia0 = np.vstack([self.inertia0, f4(inertia0)])
        self.inertia1 = np.vstack([self.inertia1, f4(inertia1)])
        self.force = np.vstack([self.force, f4((0, 0, 0, 0))])
        self.torque = np.vstack([self.torque, f4((0, 0, 0, 0))])
        self.params0 = np.vstack([self.params0, f4((smooth, drag, friction, fatten))])
        sid = self.shape_type.shape[0] - 1
        if in_scene:
            self.shape_ids = np.append(self.shape_ids, np.int32(sid)).astype(np.int32)
        return sid

    def add_sdf_block(self, dims, lower, cell: float, values: np.ndarray, header: np.ndarray | None = None):
        """Append an SDF grid (values float32 [dz,dy,dx,4]; optional header float4 placed first).

        Returns (offset, sdf_id) with the offset pointing at the header when one is given, as the
        reference stores slicer spine planes and line bounds (include/engine/geometry.h:87-101).
        """
        if self.sdf_data.shape[0] == 1 and not self.sdf_data.any():
            self.sdf_data = np.zeros((0, 4), np.float32)
            self.sdf_dims = np.zeros((0, 4), np.int32)
            self.sdf_lbcs = np.zeros((0, 4), np.float32)
        offset = self.sdf_data.shape[0]
        parts = []
        if header is not None:
            parts.append(np.asarray(header, np.float32).reshape(-1, 4))
        parts.append(np.asarray(values, np.float32).reshape(-1, 4))
        self.sdf_data = np.vstack([self.sdf_data] + parts)
        self.sdf_dims = np.vstack([self.sdf_dims, np.asarray([*dims, 0], np.int32).reshape(1, 4)])
        self.sdf_lbcs = np.vstack([self.sdf_lbcs, np.asarray([*lower, cell], np.float32).reshape(1, 4)])
        return offset, self.sdf_dims.shape[0] - 1


def int_bits(i: int) -> float:
    """A float whose bits are the integer ``i`` (the reference's CR_INT_AS_FLOAT)."""
    return float(np.array([i], np.int32).view(np.float32)[0])


@dataclasses.dataclass
class Scene:
    solver_type: int
    grid_min: np.ndarray  # float32 [3]
    grid_max: np.ndarray  # float32 [3]
    cell_size: float
    dt: float
    gravity: np.ndarray  # float32 [3]
    iterations: int
    contact_model: int
    pos_mass: np.ndarray  # float32 [N,4]
    vel: np.ndarray  # float32 [N,4]
    mat_params: np.ndarray  # float32 [N,4]
    mat_type: np.ndarray  # int32 [N]
    mask: np.ndarray  # uint8 [N]
    shapes: ShapeTable
    name: str = ""
    num_max: int = 0

    @property
    def n(self) -> int:
        return int(self.pos_mass.shape[0])

    def grid_dims(self) -> tuple[int, int, int]:
        """Node counts int((max - min) / dx + 1) evaluated in float32 (gpu_mls_mpm_solver.cu:48-49)."""
        size = (self.grid_min.astype(np.float32) * np.float32(-1) + self.grid_max.astype(np.float32))
        dims = size / np.float32(self.cell_size) + np.float32(1.0)
        return tuple(int(d) for d in dims.astype(np.float32))


def _particles(pos: np.ndarray, mass: float, mat_params, mat_type: int):
    n = pos.shape[0]
    pm = np.zeros((n, 4), np.float32)
    pm[:, :3] = pos
    pm[:, 3] = np.float32(mass)
    vel = np.zeros((n, 4), np.float32)
    mp = np.tile(np.asarray(mat_params, np.float32).reshape(1, 4), (n, 1))
    mt = np.full(n, mat_type, np.int32)
    mask = np.ones(n, np.uint8)
    return pm, vel, mp, mt, mask


def cube_drop(seed: int = 1001, side: float = 0.4, cell: float = 0.05, ppc: int = 8, E: float = 1e4,
              nu: float = 0.3, rho: float = 1000.0, dt: float = 2e-4, solver: int = SOLVER_MLS,
              material: int = MAT_NEOHOOKEAN, friction: float = 0.3) -> Scene:
    """Elastic cube dropped on a ground plane: [-1,1]^3, dx 0.05, 0.4 m cube at (0, 0.5, 0), ~4096 p."""
    lam, mu = lame(E, nu)
    h = side / 2
    pos = jittered_box((-h, 0.5 - h, -h), (h, 0.5 + h, h), cell, ppc, seed)
    mass = rho * cell ** 3 / ppc
    pm, vel, mp, mt, mask = _particles(pos, mass, (lam, mu, 0, 0), material)
    st = ShapeTable.empty()
    g = st.add_geometry(GEOM_PLANE, (0, 0, 0, 0))
    st.add_shape(g, SHAPE_STATIC, (0, 0, 0), smooth=0.0, drag=1.0, friction=friction)
    return Scene(solver, np.array([-1, -1, -1], np.float32), np.array([1, 1, 1], np.float32), cell, dt,
                 np.array([0, -9.81, 0], np.float32), 20, 0, pm, vel, mp, mt, mask, st, "cube_drop")


def tissue_slab(seed: int = 1002, size=(1.0, 0.2, 1.0), cell: float = 0.01, ppc: int = 8, E: float = 2e4,
                nu: float = 0.4, rho: float = 1050.0, dt: float = 1e-4, probe_radius: float = 0.05,
                probe_speed: float = 0.1, friction: float = 0.3, pin_thickness: float = 0.02,
                bounds_min=(-0.6, -0.1, -0.6), bounds_max=(0.6, 0.5, 0.6)) -> Scene:
    """Tissue slab with its four side faces pinned by static boxes and a kinematic sphere probe.

    Defaults are the 1.6M-particle slab: 1.0 x 0.2 x 1.0 m, dx 0.01, 8 ppc, Neo-Hookean
    E 2e4 / nu 0.4, density 1050, sphere r 0.05 descending at 0.1 m/s onto the slab centre.
    """
    lam, mu = lame(E, nu)
    sx, sy, sz = size
    pos = jittered_box((-sx / 2, 0.0, -sz / 2), (sx / 2, sy, sz / 2), cell, ppc, seed)
    mass = rho * cell ** 3 / ppc
    pm, vel, mp, mt, mask = _particles(pos, mass, (lam, mu, 0, 0), MAT_NEOHOOKEAN)
    st = ShapeTable.empty()
    # Static boxes abut the four side faces; grid nodes within one cell of a face take the box's
    # (zero) velocity because drag 0 removes all tangential motion (mpm_rigid_contact.h:356-374).
    t = pin_thickness
    gx = st.add_geometry(GEOM_BOX, (t, sy / 2 + t, sz / 2 + 2 * t, 0))
    gz = st.add_geometry(GEOM_BOX, (sx / 2 + 2 * t, sy / 2 + t, t, 0))
    for sgn in (-1.0, 1.0):
        st.add_shape(gx, SHAPE_STATIC, (sgn * (sx / 2 + t), sy / 2, 0), smooth=cell, drag=0.0, friction=0.0)
        st.add_shape(gz, SHAPE_STATIC, (0, sy / 2, sgn * (sz / 2 + t)), smooth=cell, drag=0.0, friction=0.0)
    gs = st.add_geometry(GEOM_SPHERE, (probe_radius, 0, 0, 0))
    st.add_shape(gs, SHAPE_KINEMATIC, (0, sy + probe_radius + cell, 0), smooth=0.0, drag=1.0, friction=friction,
                 lin_vel=(0, -probe_speed, 0))
    return Scene(SOLVER_MLS, np.array(bounds_min, np.float32), np.array(bounds_max, np.float32), cell, dt,
                 np.array([0, -9.81, 0], np.float32), 20, 0, pm, vel, mp, mt, mask, st, "tissue_slab")


def pb_cutting(seed: int = 1003, size=(0.6, 0.1, 0.6), cell: float = 0.008, ppc: int = 8, dt: float = 0.002,
               iterations: int = 20, relax: float = 1.0, ratio: float = 0.9, blade_speed: float = 0.2,
               depth: float = 0.05, bounds_min=(-0.4, -0.2, -0.4), bounds_max=(0.4, 0.2, 0.4)) -> Scene:
    """PB-MPM slab cut by a kinematic quad slicer blade sweeping along +x.

    PB-MPM's material params are (elastic relaxation, elasticity ratio)
    (constitutive_models.h:143-148); E and nu have no meaning there.  The slab sits on a ground
    plane and the blade is a vertical quad (local x-z plane rotated to world x-y) of half size
    0.15 x 0.025 m, as the reference's cutting example builds it (examples/example_cutting/main.cpp:96-111).
    """
    sx, sy, sz = size
    pos = jittered_box((-sx / 2, -sy, -sz / 2), (sx / 2, 0.0, sz / 2), cell, ppc, seed)
    mass = 1000.0 * cell ** 3 / ppc
    pm, vel, mp, mt, mask = _particles(pos, mass, (relax, ratio, 0, 0), MAT_NEOHOOKEAN)
    st = ShapeTable.empty()
    gp = st.add_geometry(GEOM_PLANE, (0, 0, 0, 0))
    st.add_shape(gp, SHAPE_STATIC, (0, -sy, 0), smooth=0.0, drag=1.0, friction=0.5)
    gq = st.add_geometry(GEOM_QUAD_SLICER, (0.15, 0.025, 0, 0))
    # rotate local y (blade normal) to world z: 90 degrees about x.
    c = math.cos(math.pi / 4)
    st.add_shape(gq, SHAPE_KINEMATIC, (-sx / 2 - 0.05, -depth + 0.025, 0.0), rotation=(c, 0, 0, c),
                 smooth=0.0, drag=1.0, friction=0.0, fatten=0.001, lin_vel=(blade_speed, 0, 0))
    return Scene(SOLVER_PB, np.array(bounds_min, np.float32), np.array(bounds_max, np.float32), cell, dt,
                 np.array([0, -9.81, 0], np.float32), iterations, 0, pm, vel, mp, mt, mask, st, "pb_cutting")


def batched_scenes(seed: int = 1004, num_scenes: int = 256, cells: int = 64, cell: float = 0.02, ppc: int = 8,
                   nmin: int = 2000, nmax: int = 64000, dt: float = 2e-4) -> list[Scene]:
    """Independent elastic bodies, one per scene: 64^3-cell grids, log-uniform 2k-64k particles.

    Each scene is a box of seeded dimensions resting above a ground plane with a sphere probe at a
    seeded pose; E ~ U[5e3, 5e4], nu ~ U[0.25, 0.45].
    """
    rng = np.random.default_rng(seed)
    out = []
    L = cells * cell
    for s in range(num_scenes):
        target = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
        ncell = max(target / ppc, 1.0)
        aspect = rng.uniform(0.6, 1.6, size=3)
        aspect /= aspect.prod() ** (1 / 3)
        dims = np.maximum(np.rint(aspect * ncell ** (1 / 3)), 1).astype(int)
        dims = np.minimum(dims, cells - 12)
        ext = dims * cell
        lo = np.array([-ext[0] / 2, 0.1, -ext[2] / 2])
        pos = jittered_box(lo, lo + ext, cell, ppc, seed * 1000 + s)
        E = rng.uniform(5e3, 5e4)
        nu = rng.uniform(0.25, 0.45)
        lam, mu = lame(E, nu)
        mass = 1000.0 * cell ** 3 / ppc
        pm, vel, mp, mt, mask = _particles(pos, mass, (lam, mu, 0, 0), MAT_NEOHOOKEAN)
        st = ShapeTable.empty()
        gp = st.add_geometry(GEOM_PLANE, (0, 0, 0, 0))
        st.add_shape(gp, SHAPE_STATIC, (0, 0, 0), friction=0.3)
        gs = st.add_geometry(GEOM_SPHERE, (rng.uniform(0.03, 0.08), 0, 0, 0))
        st.add_shape(gs, SHAPE_STATIC, (rng.uniform(-0.2, 0.2), 0.1 + ext[1] + rng.uniform(0.0, 0.05),
                                        rng.uniform(-0.2, 0.2)), friction=0.3)
        sc = Scene(SOLVER_MLS, np.array([-L / 2, -0.1, -L / 2], np.float32),
                   np.array([L / 2, L - 0.1, L / 2], np.float32), cell, dt, np.array([0, -9.81, 0], np.float32),
                   20, 0, pm, vel, mp, mt, mask, st, f"batch{s}")
        out.append(sc)
    return out


def material_cube(seed: int = 1005, side: float = 0.4, cell: float = 0.02, ppc: int = 8, E: float = 2e4,
                  nu: float = 0.35, rho: float = 1000.0, dt: float = 2e-4, v0=(0.0, 0.0, 0.0),
                  drop: float = 0.05) -> Scene:
    """64k-particle cube over a ground plane for material identification (dx 0.02, 20 cells/side).

    The cube's lower face starts ``drop`` above the plane and moves with initial velocity ``v0``.
    """
    lam, mu = lame(E, nu)
    h = side / 2
    pos = jittered_box((-h, drop, -h), (h, drop + side, h), cell, ppc, seed)
    mass = rho * cell ** 3 / ppc
    pm, vel, mp, mt, mask = _particles(pos, mass, (lam, mu, 0, 0), MAT_NEOHOOKEAN)
    vel[:, :3] = np.asarray(v0, np.float32)
    st = ShapeTable.empty()
    g = st.add_geometry(GEOM_PLANE, (0, 0, 0, 0))
    st.add_shape(g, SHAPE_STATIC, (0, 0, 0), friction=0.3)
    return Scene(SOLVER_MLS, np.array([-0.5, -0.1, -0.5], np.float32), np.array([0.5, 0.7, 0.5], np.float32),
                 cell, dt, np.array([0, -9.81, 0], np.float32), 20, 0, pm, vel, mp, mt, mask, st, "material_cube")


def _sphere_sdf_grid(radius: float, cell: float, margin: int = 3):
    """Sampled SDF of a sphere on a regular grid: values (float32 [dz,dy,dx,4]) and metadata."""
    n = int(math.ceil(2 * radius / cell)) + 2 * margin + 1
    lower = -(n - 1) / 2 * cell
    ax = lower + np.arange(n) * cell
    z, y, x = np.meshgrid(ax, ax, ax, indexing="ij")
    r = np.sqrt(x * x + y * y + z * z)
    vals = np.zeros((n, n, n, 4), np.float32)
    rr = np.maximum(r, 1e-9)
    vals[..., 0] = x / rr
    vals[..., 1] = y / rr
    vals[..., 2] = z / rr
    vals[..., 3] = r - radius
    return vals, (n, n, n), (lower, lower, lower)


def _plane_slicer_grid(half: float, cell: float, thickness_cells: int = 3):
    """Sampled signed distance of the plane y = 0 over a box (a flat cutting blade)."""
    nx = int(math.ceil(2 * half / cell)) + 1
    ny = 2 * thickness_cells + 1
    lower = (-(nx - 1) / 2 * cell, -thickness_cells * cell, -(nx - 1) / 2 * cell)
    vals = np.zeros((nx, ny, nx, 4), np.float32)
    ys = lower[1] + np.arange(ny) * cell
    vals[..., 1] = 1.0
    vals[..., 3] = ys[None, :, None]
    return vals, (nx, ny, nx), lower


def contact_scene(kind: str, seed: int = 1010, solver: int = SOLVER_MLS, dt: float = 2e-4) -> Scene:
    """A small cube (4096 particles) moving onto one rigid geometry of the given kind.

    kinds: box, sphere, plane, capsule, arc, lines, trimesh, quad_slicer, mesh_slicer,
    dynamic_sphere (coupling force recorded), effmass_sphere (effective-mass contact model),
    scaled_box (rotated, non-uniformly scaled box).
    """
    cell = 0.02
    h = 0.08
    pos = jittered_box((-h, 0.12 - h, -h), (h, 0.12 + h, h), cell, 8, seed)
    lam, mu = lame(2e4, 0.3)
    pm, vel, mp, mt, mask = _particles(pos, 1000.0 * cell ** 3 / 8, (lam, mu, 0, 0), MAT_NEOHOOKEAN)
    vel[:, 1] = -1.0
    st = ShapeTable.empty()
    contact_model = 0
    kin = dict(smooth=cell, drag=0.8, friction=0.3)
    if kind == "box":
        g = st.add_geometry(GEOM_BOX, (0.06, 0.02, 0.06, 0))
        st.add_shape(g, SHAPE_STATIC, (0.01, 0.0, -0.01), **kin)
    elif kind == "scaled_box":
        g = st.add_geometry(GEOM_BOX, (0.06, 0.02, 0.06, 0))
        c, s = math.cos(0.2), math.sin(0.2)
        st.add_shape(g, SHAPE_KINEMATIC, (0.0, 0.0, 0.0), rotation=(0, 0, s, c), inv_scale=(1 / 1.2, 1 / 0.8, 1.0),
                     lin_vel=(0.1, 0, 0), ang_vel=(0, 0.5, 0), **kin)
    elif kind == "sphere":
        g = st.add_geometry(GEOM_SPHERE, (0.05, 0, 0, 0))
        st.add_shape(g, SHAPE_KINEMATIC, (0.02, -0.01, 0.0), lin_vel=(0, 0.2, 0), **kin)
    elif kind == "plane":
        g = st.add_geometry(GEOM_PLANE, (0, 0, 0, 0))
        c, s = math.cos(0.15), math.sin(0.15)
        st.add_shape(g, SHAPE_STATIC, (0, 0.01, 0), rotation=(s, 0, 0, c), **kin)
    elif kind == "capsule":
        g = st.add_geometry(GEOM_CAPSULE, (0.03, 0.05, 0, 0))
        c = math.cos(math.pi / 4)
        st.add_shape(g, SHAPE_STATIC, (0, 0.0, 0), rotation=(0, 0, c, c), **kin)
    elif kind == "arc":
        g = st.add_geometry(GEOM_ARC, (-2.5, 2.5, 0, 0))
        st.add_shape(g, SHAPE_KINEMATIC, (0, 0.06, 0), inv_scale=(1 / 0.07, 1 / 0.07, 1 / 0.07), lin_vel=(0, 0.3, 0),
                     smooth=0.01, drag=1.0, friction=0.5)
    elif kind == "lines":
        pts = np.array([[-0.1, 0.06, -0.05], [-0.03, 0.07, 0.0], [0.03, 0.06, 0.02], [0.1, 0.07, 0.04]], np.float32)
        lo = pts.min(0) - 0.05
        hi = pts.max(0) + 0.05
        vals = np.zeros((len(pts), 4), np.float32)
        vals[:, :3] = pts
        header = np.array([[hi[0], hi[1], hi[2], 0]], np.float32)
        off, sid = st.add_sdf_block((0, 0, 0), lo, 0.0, vals, header=header)
        g = st.add_geometry(GEOM_CONNECTED_LINE_SEGMENTS, (int_bits(off), int_bits(sid), int_bits(len(pts) + 1), 0))
        st.add_shape(g, SHAPE_KINEMATIC, (0, 0, 0), lin_vel=(0, 0.2, 0), smooth=0.01, drag=1.0, friction=0.5)
    elif kind == "trimesh":
        vals, dims, lower = _sphere_sdf_grid(0.05, 0.01)
        off, sid = st.add_sdf_block(dims, lower, 0.01, vals)
        g = st.add_geometry(GEOM_TRIANGLE_MESH, (int_bits(off), int_bits(sid), int_bits(vals.size // 4), 0))
        st.add_shape(g, SHAPE_STATIC, (0.0, 0.0, 0.01), **kin)
    elif kind in ("quad_slicer", "mesh_slicer"):
        if kind == "quad_slicer":
            g = st.add_geometry(GEOM_QUAD_SLICER, (0.12, 0.12, 0, 0))
        else:
            vals, dims, lower = _plane_slicer_grid(0.12, 0.01)
            spine = np.array([[0.0, 0.0, 1.0, -0.5]], np.float32)  # spine where local z > 0.5 (outside)
            off, sid = st.add_sdf_block(dims, lower, 0.01, vals, header=spine)
            g = st.add_geometry(GEOM_TRIANGLE_MESH_SLICER, (int_bits(off), int_bits(sid), int_bits(vals.size // 4 + 1), 0))
        # blade normal (local y) rotated to world x: the cube is cut along x = 0.003
        c = math.cos(math.pi / 4)
        st.add_shape(g, SHAPE_KINEMATIC, (0.003, 0.12, 0.0), rotation=(0, 0, c, c), smooth=0.0, drag=1.0, friction=0.0,
                     fatten=0.002, lin_vel=(0, -0.2, 0))
        gp = st.add_geometry(GEOM_PLANE, (0, 0, 0, 0))
        st.add_shape(gp, SHAPE_STATIC, (0, 0.0, 0), **kin)
    elif kind in ("dynamic_sphere", "effmass_sphere"):
        g = st.add_geometry(GEOM_SPHERE, (0.05, 0, 0, 0))
        st.add_shape(g, SHAPE_DYNAMIC, (0.01, -0.01, 0.0), com_inv_mass=(0.0, 0.0, 0.0, 2.0),
                     inertia0=(50.0, 50.0, 50.0, 0), inertia1=(1.0, 0.5, 0.2, 0), **kin)
        contact_model = 1 if kind == "effmass_sphere" else 0
    else:
        raise ValueError(kind)
    return Scene(solver, np.array([-0.3, -0.2, -0.3], np.float32), np.array([0.3, 0.4, 0.3], np.float32), cell, dt,
                 np.array([0, -9.81, 0], np.float32), 10, contact_model, pm, vel, mp, mt, mask, st, f"contact_{kind}")


def mesh_contact_scene(dims, lower, cell: float, values=None, slicer: bool = False, spine=None, seed: int = 1012,
                       dt: float = 2e-4):
    """The contact cube of ``contact_scene`` against a triangle-mesh geometry whose SDF grid
    (``dims``, ``lower``, ``cell``; ``values`` float32 [nx*ny*nz, 4] or zeros to fill later) was
    built from a mesh: a rigid eTriangleMesh under the cube, or with ``slicer`` an
    eTriangleMeshSlicer blade in the pose of the "mesh_slicer" kind (spine plane ``spine``, stored
    one element before the grid as the reference's factory does).  Returns (scene, grid offset
    into the scene's SDF data array)."""
    cell_p = 0.02
    h = 0.08
    pos = jittered_box((-h, 0.12 - h, -h), (h, 0.12 + h, h), cell_p, 8, seed)
    lam, mu = lame(2e4, 0.3)
    pm, vel, mp, mt, mask = _particles(pos, 1000.0 * cell_p ** 3 / 8, (lam, mu, 0, 0), MAT_NEOHOOKEAN)
    vel[:, 1] = -1.0
    n = int(np.prod(dims))
    vals = np.zeros((n, 4), np.float32) if values is None else np.asarray(values, np.float32).reshape(n, 4)
    st = ShapeTable.empty()
    kin = dict(smooth=cell_p, drag=0.8, friction=0.3)
    if not slicer:
        off, sid = st.add_sdf_block(dims, lower, cell, vals)
        g = st.add_geometry(GEOM_TRIANGLE_MESH, (int_bits(off), int_bits(sid), int_bits(n), 0))
        st.add_shape(g, SHAPE_STATIC, (0.0, 0.0, 0.01), **kin)
        grid_off = off
    else:
        sp = np.asarray([(np.nan, 0.0, 0.0, 0.0) if spine is None else spine], np.float32)
        off, sid = st.add_sdf_block(dims, lower, cell, vals, header=sp)
        g = st.add_geometry(GEOM_TRIANGLE_MESH_SLICER, (int_bits(off), int_bits(sid), int_bits(n + 1), 0))
        c = math.cos(math.pi / 4)
        st.add_shape(g, SHAPE_KINEMATIC, (0.003, 0.12, 0.0), rotation=(0, 0, c, c), smooth=0.0, drag=1.0, friction=0.0,
                     fatten=0.002, lin_vel=(0, -0.2, 0))
        gp = st.add_geometry(GEOM_PLANE, (0, 0, 0, 0))
        st.add_shape(gp, SHAPE_STATIC, (0, 0.0, 0), **kin)
        grid_off = off + 1
    sc = Scene(SOLVER_MLS, np.array([-0.3, -0.2, -0.3], np.float32), np.array([0.3, 0.4, 0.3], np.float32), cell_p, dt,
               np.array([0, -9.81, 0], np.float32), 10, 0, pm, vel, mp, mt, mask, st,
               "mesh_slicer_built" if slicer else "trimesh_built")
    return sc, grid_off


# Geometry types whose params (x, y) are (offset into the SDF data, SDF id) as int bits.
_SDF_GEOMS = (GEOM_TRIANGLE_MESH, GEOM_TRIANGLE_MESH_SLICER, GEOM_CONNECTED_LINE_SEGMENTS)


def _has_sdf(st: ShapeTable) -> bool:
    return not (st.sdf_data.shape[0] == 1 and not st.sdf_data.any() and not st.sdf_dims.any())


def merge_shape_tables(tables: list[ShapeTable]) -> tuple[ShapeTable, list[int]]:
    """Concatenate shape tables into one (the layout a batch binds).

    Shapes, geometries and SDF blocks are appended table by table; geometry indices and the SDF
    offsets / ids inside SDF-backed geometry params are shifted accordingly.  Returns the merged
    table and, per input table, the offset of its shape ids in the merged shape-id list.
    """
    out = ShapeTable.empty()
    keys4 = ("position", "rotation", "inv_scale", "lin_vel", "ang_vel", "com_inv_mass", "inertia0", "inertia1",
             "force", "torque", "params0")
    sdf_dims, sdf_lbcs, sdf_data = [], [], []
    n_sdf = n_data = 0
    shape_offsets = []
    ids = []
    for st in tables:
        s0, g0 = out.shape_type.shape[0], out.geom_type.shape[0]
        gp = st.geom_params.copy()
        if _has_sdf(st):
            for gi, gt in enumerate(st.geom_type):
                if int(gt) in _SDF_GEOMS:
                    off, sid = gp[gi, :2].view(np.int32)
                    gp[gi, 0] = int_bits(int(off) + n_data)
                    gp[gi, 1] = int_bits(int(sid) + n_sdf)
            sdf_dims.append(st.sdf_dims)
            sdf_lbcs.append(st.sdf_lbcs)
            sdf_data.append(st.sdf_data)
            n_sdf += st.sdf_dims.shape[0]
            n_data += st.sdf_data.shape[0]
        out.geom_type = np.concatenate([out.geom_type, st.geom_type]).astype(np.int32)
        out.geom_params = np.vstack([out.geom_params, gp]).astype(np.float32)
        out.shape_type = np.concatenate([out.shape_type, st.shape_type]).astype(np.int32)
        out.geom_idx = np.concatenate([out.geom_idx, st.geom_idx + g0]).astype(np.int32)
        for k in keys4:
            setattr(out, k, np.vstack([getattr(out, k), getattr(st, k)]).astype(np.float32))
        shape_offsets.append(sum(len(i) for i in ids))
        ids.append(st.shape_ids + s0)
    out.shape_ids = np.concatenate(ids).astype(np.int32) if ids else np.zeros(0, np.int32)
    if sdf_dims:
        out.sdf_dims = np.vstack(sdf_dims).astype(np.int32)
        out.sdf_lbcs = np.vstack(sdf_lbcs).astype(np.float32)
        out.sdf_data = np.vstack(sdf_data).astype(np.float32)
    return out, shape_offsets


@dataclasses.dataclass
class Batch:
    """Scenes laid out for one batch solver: concatenated particles and shapes plus, per scene,
    the descriptor fields of CrB200BatchSceneDesc."""

    scenes: list
    merged: Scene  # concatenated particle arrays and the merged shape table
    particle_offset: np.ndarray  # uint32 [S]
    shape_offset: np.ndarray  # int32 [S]

    @property
    def num_scenes(self) -> int:
        return len(self.scenes)

    def slice(self, s: int) -> slice:
        o = int(self.particle_offset[s])
        return slice(o, o + self.scenes[s].n)


def make_batch(scene_list: list[Scene]) -> Batch:
    """Lay out scenes of one solver type back to back (particles in scene order)."""
    if not scene_list:
        raise ValueError("a batch needs at least one scene")
    t = scene_list[0].solver_type
    it = scene_list[0].iterations
    if any(s.solver_type != t or s.iterations != it for s in scene_list):
        raise ValueError("the scenes of a batch share the solver type and iteration count")
    offs = np.cumsum([0] + [s.n for s in scene_list[:-1]]).astype(np.uint32)
    shapes, soffs = merge_shape_tables([s.shapes for s in scene_list])
    cat = lambda k: np.concatenate([getattr(s, k) for s in scene_list])  # noqa: E731
    s0 = scene_list[0]
    merged = Scene(t, s0.grid_min, s0.grid_max, s0.cell_size, s0.dt, s0.gravity, it, s0.contact_model,
                   cat("pos_mass"), cat("vel"), cat("mat_params"), cat("mat_type"), cat("mask"), shapes, "batch")
    return Batch(list(scene_list), merged, offs, np.asarray(soffs, np.int32))


def adjoint_scene(kind: str = "plane", seed: int = 1006, side: float = 0.1, cell: float = 0.02,
                  v0=(0.3, -1.5, 0.2), E: float = 2e4, nu: float = 0.35) -> Scene:
    """A 1000-particle Neo-Hookean cube 5 mm above the ground moving at v0, for gradient checks.

    kind "plane": the ground plane only.  kind "mixed": the plane, a kinematic sphere (translating
    and spinning), a static box and a tilted static capsule around the impact point, with smoothing
    distances and drags that put grid nodes in every contact branch.  kind "effmass": the
    effective-mass contact model, the plane and a rotated, moving dynamic sphere with mass and
    inertia next to the impact point (two-body impulses with friction, both friction branches).
    """
    sc = material_cube(seed=seed, side=side, cell=cell, E=E, nu=nu, v0=v0, drop=0.005)
    if kind == "mixed":
        st = ShapeTable.empty()
        g = st.add_geometry(GEOM_PLANE, (0, 0, 0, 0))
        st.add_shape(g, SHAPE_STATIC, (0, 0, 0), friction=0.3)
        g = st.add_geometry(GEOM_SPHERE, (0.04, 0, 0, 0))
        st.add_shape(g, SHAPE_KINEMATIC, (0.03, -0.02, 0.0), smooth=0.02, drag=0.8, friction=0.3,
                     lin_vel=(0, 0.2, 0), ang_vel=(0, 1.0, 0.5))
        g = st.add_geometry(GEOM_BOX, (0.03, 0.02, 0.03, 0))
        st.add_shape(g, SHAPE_STATIC, (-0.04, -0.005, 0.02), smooth=0.02, drag=0.9, friction=0.4)
        g = st.add_geometry(GEOM_CAPSULE, (0.015, 0.03, 0, 0))
        c, s_ = math.cos(0.6), math.sin(0.6)
        st.add_shape(g, SHAPE_STATIC, (0.0, 0.0, -0.04), rotation=(s_, 0, 0, c), smooth=0.02, drag=0.9, friction=0.2)
        sc.shapes = st
    elif kind == "effmass":
        st = ShapeTable.empty()
        g = st.add_geometry(GEOM_PLANE, (0, 0, 0, 0))
        st.add_shape(g, SHAPE_STATIC, (0, 0, 0), friction=0.3)
        g = st.add_geometry(GEOM_SPHERE, (0.04, 0, 0, 0))
        c, s_ = math.cos(0.4), math.sin(0.4)
        st.add_shape(g, SHAPE_DYNAMIC, (0.035, -0.015, 0.01), rotation=(0, s_, 0, c), smooth=0.02, drag=0.7,
                     friction=0.4, lin_vel=(0, 0.1, 0), ang_vel=(0.5, 0, 1.0), com_inv_mass=(0.01, 0.0, -0.005, 4.0),
                     inertia0=(300.0, 250.0, 200.0, 0), inertia1=(10.0, 5.0, 2.0, 0))
        sc.shapes = st
        sc.contact_model = 1
    elif kind != "plane":
        raise ValueError(kind)
    sc.name = f"adjoint_{kind}"
    return sc
