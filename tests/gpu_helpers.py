"""Helpers shared by the parity tests."""
import numpy as np


def rel_pos_err(x, x_ref, x0, dx):
    """max_p |x - x_ref| / max(max_p |x_ref - x0|, dx): the position tolerance metric."""
    scale = max(float(np.abs(x_ref - x0).max()), dx)
    return float(np.abs(x - x_ref).max()) / scale


def block_keys(scene, pos_xyz):
    """Cell keys exactly as the engine defines them (block-major 4x4x4 blocks of clamped base
    cells), computed from float32 positions in numpy (IEEE single, no fused multiply-add)."""
    nx, ny, nz = scene.grid_dims()
    n = np.array([nx, ny, nz])
    nb = (n + 5) >> 2
    inv = np.float32(1) / np.float32(scene.cell_size)
    sp = (pos_xyz.astype(np.float32) - scene.grid_min.astype(np.float32)) * inv
    b = np.trunc(sp - np.float32(0.5)).astype(np.int64)
    c = np.clip(b, 0, n - 2)
    blk = (c[:, 0] >> 2) + nb[0] * ((c[:, 1] >> 2) + nb[1] * (c[:, 2] >> 2))
    loc = (c[:, 0] & 3) + 4 * ((c[:, 1] & 3) + 4 * (c[:, 2] & 3))
    return (blk * 64 + loc).astype(np.uint32)


def canonical_permutation(keys, active):
    ids = np.nonzero(active)[0]
    order = np.lexsort((ids, keys[ids]))
    return ids[order].astype(np.uint32)


def factory_oracle_scene(scene, x0):
    """The factory cube (oracle/factory_run.py) as a scene for the FP64 oracle, from the particles
    the reference's sampler made."""
    from crmpm_b200 import scenes

    n = x0.shape[0]
    lam, mu = scenes.lame(1e4, 0.3)
    mp = np.tile(np.array([lam, mu, 0, 0] if scene != "cube_pb" else [1.0, 0.9, 0, 0], np.float32), (n, 1))
    st = scenes.ShapeTable.empty()
    g = st.add_geometry(scenes.GEOM_PLANE, (0, 0, 0, 0))
    st.add_shape(g, scenes.SHAPE_STATIC, (0, 0, 0), smooth=0.0, drag=1.0, friction=0.3)
    solver = {"cube_mls": scenes.SOLVER_MLS, "cube_pb": scenes.SOLVER_PB, "cube_standard": scenes.SOLVER_STANDARD}[scene]
    return scenes.Scene(solver, np.array([-0.3, -0.1, -0.3], np.float32), np.array([0.3, 0.4, 0.3], np.float32), 0.01,
                        2e-4, np.array([0.05, -9.81, 0.03], np.float32), 10, 0, x0.astype(np.float32),
                        np.zeros((n, 4), np.float32), mp, np.full(n, scenes.MAT_NEOHOOKEAN, np.int32),
                        np.ones(n, np.uint8), st, "factory_" + scene)
