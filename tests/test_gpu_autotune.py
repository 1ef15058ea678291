"""Launch-shape autotuner (CrB200SolverAutotune): it leaves the particle state untouched, and a
tuned solver's substeps match an untuned one's within the parity tolerance (launch shapes change
only the order of float atomics)."""
import numpy as np
import pytest

from conftest import cuda_available
from gpu_helpers import rel_pos_err

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

import crmpm_b200 as cb  # noqa: E402
from crmpm_b200 import scenes  # noqa: E402


@pytest.mark.parametrize("batch", [False, True])
def test_autotune_keeps_state_and_results(batch):
    cb.build_library()
    if batch:
        sl = scenes.batched_scenes(num_scenes=3, nmin=1500, nmax=4000)
        tuned, plain = cb.DeviceBatch(sl), cb.DeviceBatch(sl)
        sc = tuned.scene
    else:
        sc = scenes.cube_drop()
        tuned, plain = cb.DeviceScene(sc), cb.DeviceScene(sc)
    tuned.step(5)
    plain.step(5)
    before = tuned.state()
    choice = tuned.solver.autotune(4)
    assert choice[0] in (4, 8, 16) and choice[1] in (1, 2) and choice[2] in (1, 2)
    after = tuned.state()
    for k in ("x", "v", "F", "C"):
        np.testing.assert_array_equal(after[k], before[k])
    tuned.step(60)
    plain.step(60)
    a, b = tuned.state(), plain.state()
    assert rel_pos_err(a["x"], b["x"], sc.pos_mass[:, :3], sc.cell_size) <= 1e-4
