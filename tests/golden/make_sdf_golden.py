"""Generates tests/golden/meshsdf_*.npz: SDF grids of small procedural meshes made by the
reference's own SdfBuilder (src/geometry_utils/sdf_builder.cpp, compiled for the host as
oracle/_ref/libref_sdf.so by `make -C oracle ref`).

    python tests/golden/make_sdf_golden.py

Each fixture holds the mesh and the builder arguments next to the reference's grid, so the tests
need neither the reference sources nor the mesh generators' exact behaviour.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "cressim-mpm_b200"))

import oracle_py as op  # noqa: E402
from crmpm_b200 import meshes  # noqa: E402

NAN_SPINE = (np.nan, 0.0, 0.0, 0.0)


def cases():
    box = meshes.box((0.3, 0.2, 0.25), divisions=2)
    yield "box", box, 0.05, 0.05, True, False, NAN_SPINE
    yield "box_unnormalized", box, 0.05, 0.05, False, False, NAN_SPINE
    # away from the origin: the reference's grid still reaches back to it
    yield "box_offset", meshes.box((0.2, 0.15, 0.1), center=(0.45, 0.1, -0.3)), 0.05, 0.0, True, False, NAN_SPINE
    yield "sphere", meshes.icosphere(0.3, 2), 0.04, 0.05, True, False, NAN_SPINE
    yield "torus", meshes.torus(0.3, 0.1, 24, 12), 0.04, 0.04, True, False, NAN_SPINE
    blade = meshes.blade()
    yield "blade_slicer", blade, 0.004, 0.01, True, True, NAN_SPINE
    yield "blade_slicer_spine", blade, 0.004, 0.01, True, True, (0.0, 1.0, 0.0, -0.005)


def main():
    op.build(ref=True)
    assert op.ref_sdf_available(), "oracle/_ref/libref_sdf.so was not built"
    for name, (P, T), cell, fatten, normalize, slicer, spine in cases():
        dims, lower, grid = op.ref_sdf(P, T, cell, fatten, normalize=normalize, slicer=slicer,
                                       spine=None if np.isnan(spine[0]) else spine)
        path = os.path.join(HERE, f"meshsdf_{name}.npz")
        np.savez_compressed(path, points=P, triangles=T, cell=np.float32(cell), fatten=np.float32(fatten),
                            normalize=np.int32(normalize), slicer=np.int32(slicer), spine=np.asarray(spine, np.float32),
                            dims=np.asarray(dims, np.int32), lower=lower, grid=grid)
        print(f"{path}: dims {dims}, {len(T)} triangles")


if __name__ == "__main__":
    main()
