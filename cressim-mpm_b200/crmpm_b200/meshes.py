"""Procedural triangle meshes (float32 points [P, 3], uint32 triangles [T, 3], counter-clockwise
seen from outside) for SDF grids built with ``crmpm_b200.build_sdf``: closed surfaces for
rigid bodies (the reference's eTriangleMesh geometry) and open sheets for mesh slicers
(eTriangleMeshSlicer).  The reference loads such meshes from files; these stand in for them.
"""
from __future__ import annotations

import numpy as np


def _pack(points, tris):
    return np.ascontiguousarray(points, np.float32), np.ascontiguousarray(tris, np.uint32)


def icosphere(radius: float = 0.5, subdivisions: int = 2, center=(0.0, 0.0, 0.0)):
    """Closed sphere: an icosahedron split `subdivisions` times (20 * 4**s triangles)."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    pts = [np.asarray(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        mid = {}

        def m(a, b):
            k = (min(a, b), max(a, b))
            if k not in mid:
                p = pts[a] + pts[b]
                pts.append(p / np.linalg.norm(p))
                mid[k] = len(pts) - 1
            return mid[k]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    P = np.asarray(pts) * radius + np.asarray(center, np.float64)
    return _pack(P, faces)


def torus(major: float = 0.4, minor: float = 0.15, nu: int = 32, nv: int = 16, center=(0.0, 0.0, 0.0)):
    """Closed torus around the z axis (2 * nu * nv triangles): a non-convex body with a hole."""
    u = 2 * np.pi * np.arange(nu) / nu
    w = 2 * np.pi * np.arange(nv) / nv
    U, W = np.meshgrid(u, w, indexing="ij")
    r = major + minor * np.cos(W)
    P = np.stack([r * np.cos(U), r * np.sin(U), minor * np.sin(W)], -1).reshape(-1, 3) + np.asarray(center)
    tris = []
    for i in range(nu):
        for j in range(nv):
            a, b = i * nv + j, ((i + 1) % nu) * nv + j
            c, d = ((i + 1) % nu) * nv + (j + 1) % nv, i * nv + (j + 1) % nv
            tris += [(a, b, c), (a, c, d)]
    return _pack(P, tris)


def box(half=(0.5, 0.5, 0.5), center=(0.0, 0.0, 0.0), divisions: int = 1):
    """Closed axis-aligned box, each face split into divisions x divisions quads."""
    hx, hy, hz = half
    n = divisions
    pts, tris = [], []
    index = {}

    def vid(p):
        k = tuple(np.round(p, 9))
        if k not in index:
            index[k] = len(pts)
            pts.append(p)
        return index[k]

    s = np.linspace(-1.0, 1.0, n + 1)
    # (axis, sign): outward normal along +-axis; (u, v) spans the face counter-clockwise from outside
    for axis in range(3):
        for sign in (1.0, -1.0):
            u_ax, v_ax = (axis + 1) % 3, (axis + 2) % 3
            if sign < 0:
                u_ax, v_ax = v_ax, u_ax
            for i in range(n):
                for j in range(n):
                    q = []
                    for di, dj in ((0, 0), (1, 0), (1, 1), (0, 1)):
                        p = np.zeros(3)
                        p[axis] = sign
                        p[u_ax] = s[i + di]
                        p[v_ax] = s[j + dj]
                        q.append(vid(p * np.asarray(half) + np.asarray(center)))
                    tris += [(q[0], q[1], q[2]), (q[0], q[2], q[3])]
    return _pack(np.asarray(pts), tris)


def blade(length: float = 0.12, height: float = 0.04, camber: float = 0.01, nu: int = 12, nv: int = 4,
          center=(0.0, 0.0, 0.0)):
    """Open curved sheet in the x-y plane bowed along z (2 * nu * nv triangles): a mesh slicer
    blade with boundary edges all round."""
    x = np.linspace(-length / 2, length / 2, nu + 1)
    y = np.linspace(-height / 2, height / 2, nv + 1)
    X, Y = np.meshgrid(x, y, indexing="ij")
    Z = camber * (1.0 - (2.0 * X / length) ** 2)
    P = np.stack([X, Y, Z], -1).reshape(-1, 3) + np.asarray(center)
    tris = []
    for i in range(nu):
        for j in range(nv):
            a, b = i * (nv + 1) + j, (i + 1) * (nv + 1) + j
            c, d = (i + 1) * (nv + 1) + j + 1, i * (nv + 1) + j + 1
            tris += [(a, b, c), (a, c, d)]
    return _pack(P, tris)
