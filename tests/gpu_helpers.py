"""Helpers shared by the GPU parity tests."""
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
