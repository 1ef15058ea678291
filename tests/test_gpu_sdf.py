"""GPU triangle-mesh SDF builder (CrB200SdfCompute / CrB200SdfComputeMod) against the CPU
restatement (oracle/sdf_oracle.cpp), the reference's own grids (tests/golden/meshsdf_*.npz, made
by the reference's SdfBuilder) and, at full size, the analytic distance of the surface the mesh
approximates.

Bars: against the restatement, which runs the same single-precision operations in the same
order, bit-identical grids (distance, gradient, NaN pattern); against the reference, the bar of
tests/test_sdf_oracle.py (identical dimensions, signs and off-mesh nodes; distances within 1e-7
and bit-identical at >= 97 % of the nodes; gradients bit-identical where the distance stencil is).
"""
import os

import numpy as np
import pytest

from conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

import crmpm_b200 as cb  # noqa: E402
import oracle_py as op  # noqa: E402
from crmpm_b200 import meshes, scenes  # noqa: E402
from gpu_helpers import rel_pos_err  # noqa: E402
from test_sdf_oracle import CASES, assert_grid_matches, load  # noqa: E402


def _gpu(kw):
    cb.build_library()
    g = cb.build_sdf(kw["points"], kw["triangles"], kw["cell"], kw["fatten"], normalize=kw["normalize"],
                     slicer=kw["slicer"], spine=kw["spine"])
    import torch

    torch.cuda.synchronize()
    return g


@pytest.mark.parametrize("case", CASES)
def test_gpu_sdf_matches_restatement_bitwise(case):
    kw, _ = load(case)
    g = _gpu(kw)
    dims, lower, size, ref = op.port_sdf(**kw)
    assert g.dims == dims
    np.testing.assert_array_equal(np.asarray(g.lower, np.float32), lower)
    got = g.host()
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    np.testing.assert_array_equal(got[~np.isnan(ref)], ref[~np.isnan(ref)])


@pytest.mark.parametrize("case", CASES)
def test_gpu_sdf_matches_reference_grid(case):
    kw, z = load(case)
    g = _gpu(kw)
    assert g.dims == tuple(int(v) for v in z["dims"])
    assert_grid_matches(g.host(), z["grid"], g.dims)


def test_gpu_sdf_irregular_meshes_match_restatement_and_reference():
    rng = np.random.default_rng(5)
    P, T = meshes.torus(0.3, 0.12, 20, 10)
    P = P + (0.01 * rng.standard_normal(P.shape)).astype(np.float32)
    kw = dict(points=P, triangles=T, cell=0.03, fatten=0.05, normalize=True, slicer=False, spine=None)
    got = _gpu(kw).host()
    dims, _, _, port = op.port_sdf(**kw)
    np.testing.assert_array_equal(got, port)
    if op.ref_sdf_available():
        _, _, ref = op.ref_sdf(P, T, 0.03, 0.05)
        assert_grid_matches(got, ref, dims)
    B, TB = meshes.blade(0.1, 0.03, 0.008, 10, 3)
    B = B + (0.0005 * rng.standard_normal(B.shape)).astype(np.float32)
    kw = dict(points=B, triangles=TB, cell=0.004, fatten=0.008, normalize=True, slicer=True, spine=(0.0, 1.0, 0.1, -0.004))
    got = _gpu(kw).host()
    dims, _, _, port = op.port_sdf(**kw)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(port))
    np.testing.assert_array_equal(got[~np.isnan(port)], port[~np.isnan(port)])
    if op.ref_sdf_available():
        _, _, ref = op.ref_sdf(B, TB, 0.004, 0.008, slicer=True, spine=kw["spine"])
        assert_grid_matches(got, ref, dims, sticky_frac=0.005)


def test_gpu_sdf_full_size_sphere_against_analytic_distance():
    """5120-triangle icosphere of radius 0.3 on a 0.005 grid (about 2.5 M nodes): every distance
    is within the mesh's deviation from the sphere (its sagitta: r minus the smallest distance
    from the centre to a triangle's plane) of |x - c| - r, inside nodes are negative, and
    normalised gradients point along the radius."""
    import torch

    r, c = 0.3, np.array([0.02, -0.01, 0.03])
    P, T = meshes.icosphere(r, 4, center=tuple(c))
    cb.build_library()
    g = cb.build_sdf(P, T, 0.005, 0.04)
    torch.cuda.synchronize()
    nx, ny, nz = g.dims
    assert nx * ny * nz > 2_000_000
    grid = g.data.double()
    lo = torch.tensor(g.lower, dtype=torch.float64, device=grid.device)
    z, y, x = torch.meshgrid(*(torch.arange(n, device=grid.device, dtype=torch.float64) for n in (nz, ny, nx)),
                             indexing="ij")
    pts = torch.stack([x, y, z], -1) * np.float32(g.cell) + lo
    rad = (pts - torch.tensor(c, device=grid.device)).norm(dim=-1)
    exact = rad - r
    w = grid[..., 3]
    A, B, C_ = (P[T[:, k]].astype(np.float64) for k in range(3))
    nrm = np.cross(B - A, C_ - A)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    sag = r - float(np.abs(((A - c) * nrm).sum(1)).min())
    assert 0 < sag < 1e-3
    assert float((w - exact).abs().max()) <= sag + 1e-6
    far = exact.abs() > sag + 1e-6
    assert bool(((w < 0) == (exact < 0))[far].all())
    sel = (exact.abs() > 4 * g.cell) & (rad > 8 * g.cell)
    radial = (pts - torch.tensor(c, device=grid.device)) / rad[..., None]
    cosang = (grid[..., :3] * radial).sum(-1)
    assert float(cosang[sel].min()) > 0.99


def _scene_pair(slicer):
    if not slicer:
        P, T = meshes.icosphere(0.05, 2)
        kw = dict(cell=0.01, fatten=0.03)
        spine = None
    else:
        P, T = meshes.blade(0.24, 0.24, 0.0, 8, 8)
        P = np.ascontiguousarray(P[:, [0, 2, 1]])  # the sheet in the local x-z plane, normal local y
        T = np.ascontiguousarray(T[:, [0, 2, 1]])
        kw = dict(cell=0.01, fatten=0.03)
        spine = (0.0, 0.0, 1.0, -0.5)
    return P, T, kw, spine


@pytest.mark.parametrize("slicer", [False, True], ids=["trimesh", "mesh_slicer"])
def test_gpu_built_sdf_drives_contact_like_the_reference_built_one(slicer):
    """The factory flow: the grid is built on the GPU straight into the scene's device SDF array
    (as the reference's createGeometry writes its host array) and the contact substeps run on it.
    The same scene with the reference-built grid (the restatement stands in when the reference is
    absent) must give the same particles within the parity tolerance."""
    import torch

    P, T, kw, spine = _scene_pair(slicer)
    d = cb.sdf_desc(P, T, kw["cell"], kw["fatten"], spine)
    dims = tuple(int(v) for v in d.sdfDimension)
    lower = tuple(float(v) for v in d.lowerBound)
    n = int(np.prod(dims))
    if op.ref_sdf_available():
        _, _, ref = op.ref_sdf(P, T, kw["cell"], kw["fatten"], slicer=slicer, spine=spine)
    else:
        _, _, _, ref = op.port_sdf(P, T, kw["cell"], kw["fatten"], slicer=slicer, spine=spine)
    sc_ref, _ = scenes.mesh_contact_scene(dims, lower, kw["cell"], ref, slicer=slicer, spine=spine)
    sc_gpu, off = scenes.mesh_contact_scene(dims, lower, kw["cell"], None, slicer=slicer, spine=spine)
    cb.build_library()
    ds = cb.DeviceScene(sc_gpu)
    cb.build_sdf(P, T, kw["cell"], kw["fatten"], slicer=slicer, spine=spine, out=ds.sh["sdf_data"][off:off + n])
    torch.cuda.synchronize()
    built = ds.sh["sdf_data"][off:off + n].cpu().numpy()
    assert_grid_matches(built, ref, dims, sticky_frac=0.005 if slicer else 0.0)
    ds.step(80)
    got = ds.state()
    dr = cb.DeviceScene(sc_ref)
    dr.step(80)
    exp = dr.state()
    e = rel_pos_err(got["x"], exp["x"], sc_ref.pos_mass[:, :3], sc_ref.cell_size)
    assert e <= 1e-4, e
    moved = np.abs(exp["x"] - sc_ref.pos_mass[:, :3]).max()
    assert moved > 0.01  # the bodies did meet


ADAPTER_CHECK = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                             "sdf_adapter_check")


@pytest.mark.skipif(not os.path.exists(ADAPTER_CHECK), reason="oracle/_ref/sdf_adapter_check not built")
@pytest.mark.parametrize("slicer", [False, True], ids=["trimesh", "mesh_slicer"])
def test_reference_side_adapter_matches_reference_builder(slicer, tmp_path):
    """The drop-in for the factory (adapter/gpu_b200_sdf_builder.h) run against the reference's
    own SdfBuilder in one program, as createGeometry would call them: same descriptor, same off-mesh
    nodes (up to the reference's order-dependent slicer flag), signs equal, distances within 1e-7."""
    import subprocess

    if slicer:
        P, T = meshes.blade(0.1, 0.04, 0.01, 10, 4)
        cell, fatten = 0.004, 0.01
    else:
        P, T = meshes.torus(0.25, 0.08, 24, 12)
        cell, fatten = 0.02, 0.04
    path = tmp_path / "mesh.bin"
    with open(path, "wb") as f:
        np.asarray([len(P), len(T)], np.int32).tofile(f)
        np.ascontiguousarray(P, np.float32).tofile(f)
        np.ascontiguousarray(T, np.uint32).tofile(f)
    r = subprocess.run([ADAPTER_CHECK, str(path), str(cell), str(fatten), str(int(slicer))], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    f = dict(zip(r.stdout.split()[0::2], r.stdout.split()[1::2]))
    nodes = int(f["nodes"])
    assert int(f["desc_same"]) == 1
    assert int(f["sign_differ"]) == 0
    assert float(f["maxdiff"]) <= 1e-7
    assert int(f["differ"]) <= 0.03 * nodes
    assert int(f["nan_differ"]) <= 0.005 * nodes
