"""The factory driver on the reference's CPU path (no GPU): oracle/factory_run.py with --cpu makes
the reference's factory (oracle/build_factory.sh, the unchanged build) fall back to its CPU solvers,
whose arithmetic the oracle restates.  The cube run through CrCreateScene / CrAdvance /
CrFetchResults must then equal the oracle's float32 restatement of the same scene to rounding,
which pins the scene the GPU factory tests rebuild for their FP64 runs (tests/test_gpu_factory.py)
and the count of substeps SceneImpl takes per frame."""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle_py as op

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "factory", "libcrmpm_factory_ref.so")


@pytest.mark.skipif(not os.path.exists(LIB), reason="oracle/_ref/factory not built (make -C oracle ref-factory)")
@pytest.mark.parametrize("scene", ["cube_mls", "cube_standard"])
def test_factory_cpu_path_equals_the_oracle(scene, tmp_path):
    from gpu_helpers import factory_oracle_scene

    out = str(tmp_path / "f.npz")
    frames = 3
    r = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "factory_run.py"), LIB, scene, str(frames), out,
                        "1.0", "--cpu"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    d = dict(np.load(out))
    # 10 x dt accumulated in float is one substep short of the frame: SceneImpl takes 11
    assert int(d["substeps"]) == 11
    o = op.PortOracle(factory_oracle_scene(scene, d["x0"]), 32)
    o.compute_initial_data()
    o.step(frames * int(d["substeps"]))
    st = o.state()
    assert float(np.abs(d["x"][:, :3] - st["x"]).max()) <= 1e-7
    assert float(np.abs(d["v"][:, :3] - st["v"]).max()) <= 1e-5
