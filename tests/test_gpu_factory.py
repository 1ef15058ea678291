"""The whole reference factory with the engine dropped in: the reference's engine and C API built
from its own sources three ways (oracle/build_factory.sh: as it is; with createScene's solver
switch constructing the engine's adapters; and also with SceneImpl reading back only the allocated
particles), each scene run through CrCreateScene / CrAdvance / CrFetchResults
(c_api/include/crmpm_c_api.h:141-176) in its own process (oracle/factory_run.py).

The drop-in must give what the reference's own CUDA solver gives through the same factory:
positions within 1e-4 of max(displacement, dx) for MLS and standard MPM and 2e-3 for PB-MPM (the
bars of the engine-vs-reference-CUDA tests), velocities within 1e-3 of their scale, the coupling
force and torque within 1e-3.  The slab run also times CrAdvance + CrFetchResults per frame of 10
substeps in all three builds, with numMaxParticles twice the allocated particles so that the
readback change shows.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FACT = os.path.join(ROOT, "oracle", "_ref", "factory")
LIBS = {k: os.path.join(FACT, f"libcrmpm_factory_{k}.so") for k in ("ref", "b200", "b200_rb")}
built = all(os.path.exists(p) for p in LIBS.values())


def _run(kind, scene, frames, tmp_path, spare=1.0):
    out = str(tmp_path / f"{kind}_{scene}.npz")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "factory_run.py"), LIBS[kind], scene, str(frames),
                        out, str(spare)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return dict(np.load(out))


def _compare(a, b, tol, what):
    x0 = b["x0"][:, :3]
    scale = max(float(np.abs(b["x"][:, :3] - x0).max()), 0.01)
    e = float(np.abs(a["x"][:, :3] - b["x"][:, :3]).max()) / scale
    vscale = max(float(np.abs(b["v"][:, :3]).max()), 1e-3)
    ev = float(np.abs(a["v"][:, :3] - b["v"][:, :3]).max()) / vscale
    cscale = max(float(np.abs(b["coupling"]).max()), 1e-6)
    ec = float(np.abs(a["coupling"] - b["coupling"]).max()) / cscale
    print(f"FACTORY {what} n={int(b['n'])} e_x={e:.3e} tol={tol:.0e} e_v={ev:.3e} e_coupling={ec:.3e} "
          f"disp={scale:.3e}")
    np.testing.assert_array_equal(a["x0"], b["x0"])
    assert e <= tol, f"{what}: positions {e:.3e} > {tol:.0e}"
    assert ev <= 1e-3, f"{what}: velocities {ev:.3e}"
    assert ec <= 1e-3, f"{what}: coupling {ec:.3e}"


@pytest.mark.skipif(not built, reason="oracle/_ref/factory not built (make -C oracle ref-factory)")
@pytest.mark.parametrize("scene,frames,tol", [("cube_mls", 40, 1e-4), ("cube_standard", 40, 1e-4), ("cube_pb", 40, 2e-3)])
def test_factory_cube_through_the_c_api(scene, frames, tol, tmp_path):
    ref = _run("ref", scene, frames, tmp_path)
    got = _run("b200", scene, frames, tmp_path)
    assert float(np.abs(ref["x"][:, :3] - ref["x0"][:, :3]).max()) > 1e-3, "the cube did not move"
    _compare(got, ref, tol, scene)
    # a small scene shows the host cost a frame adds (10 substeps, the adapter's C-ABI calls)
    print(f"FACTORY {scene} frame ms (10 substeps): reference {np.median(ref['times'][1:]) * 1e3:.3f}, "
          f"drop-in {np.median(got['times'][1:]) * 1e3:.3f}")


@pytest.mark.skipif(not built, reason="oracle/_ref/factory not built (make -C oracle ref-factory)")
def test_factory_slab_through_the_c_api_and_its_frame_time(tmp_path):
    frames = 4
    ref = _run("ref", "slab", frames, tmp_path, spare=2.0)
    got = _run("b200", "slab", frames, tmp_path, spare=2.0)
    rb = _run("b200_rb", "slab", frames, tmp_path, spare=2.0)
    _compare(got, ref, 1e-4, "slab")
    _compare(rb, got, 1e-4, "slab readback")
    # frame times after the first (which holds initialisation and the first-touch allocations)
    t = {k: float(np.median(d["times"][1:])) * 1e3 for k, d in (("ref", ref), ("b200", got), ("b200_rb", rb))}
    print(f"FACTORY slab frame ms (10 substeps, CrAdvance + CrFetchResults): reference {t['ref']:.3f}, "
          f"drop-in {t['b200']:.3f}, drop-in with active-range readback {t['b200_rb']:.3f}")
    assert t["b200"] < t["ref"]
