"""Batch sharding across ranks, world size 2 over gloo.

Each rank takes its scenes from shard_scenes, steps them, and rank 0 gathers the results: the
union covers every scene exactly once, loads are balanced within one scene, and the positions equal
those of one process stepping all scenes (scenes are independent, so sharding changes no result).
The CPU test steps the CPU oracle; the GPU test steps the engine's batch solver in each rank.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import cuda_available
from crmpm_b200 import scenes
from crmpm_b200.sharding import shard_loads, shard_scenes


def test_shard_balance_and_cover():
    rng = np.random.default_rng(0)
    counts = np.exp(rng.uniform(np.log(2000), np.log(64000), 256)).astype(int)
    for world in (1, 2, 3, 8):
        sh = shard_scenes(counts, world)
        flat = sorted(s for r in sh for s in r)
        assert flat == list(range(256))
        loads = shard_loads(counts, sh)
        assert max(loads) - min(loads) <= counts.max()
    assert shard_scenes([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]


def _scene_list():
    return scenes.batched_scenes(seed=21, num_scenes=5, cells=24, nmin=200, nmax=600)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import sys

    import torch.distributed as dist

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [os.path.join(here, "..", "oracle"), os.path.join(here, "..", "cressim-mpm_b200")]
    import oracle_py as op

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sl = _scene_list()
    mine = shard_scenes([sc.n for sc in sl], world)[rank]
    res = {}
    for s in mine:
        o = op.PortOracle(sl[s], 32)
        o.compute_initial_data()
        o.step(3)
        res[s] = o.state()["x"]
    gathered = [None] * world
    dist.all_gather_object(gathered, res)
    if rank == 0:
        merged = {}
        for g in gathered:
            assert not set(g) & set(merged)
            merged.update(g)
        np.savez(os.path.join(out_dir, "sharded.npz"), **{str(k): v for k, v in merged.items()})
    dist.destroy_process_group()


def test_sharded_batch_equals_single_process(tmp_path):
    import oracle_py as op

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    got = np.load(tmp_path / "sharded.npz")
    sl = _scene_list()
    assert sorted(int(k) for k in got.files) == list(range(len(sl)))
    for s, sc in enumerate(sl):
        o = op.PortOracle(sc, 32)
        o.compute_initial_data()
        o.step(3)
        np.testing.assert_array_equal(got[str(s)], o.state()["x"])


def _engine_rank_main(rank, world, port, out_dir, steps):
    """One rank of the engine-in-the-loop run: a DeviceBatch of this rank's scenes on cuda:0, its
    substeps, and the positions and velocities gathered to rank 0 over gloo (host memory; the ranks'
    kernels never wait on one another)."""
    import sys

    import torch.distributed as dist

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [os.path.join(here, "..", "oracle"), os.path.join(here, "..", "cressim-mpm_b200")]
    import crmpm_b200 as cb
    from crmpm_b200 import scenes as sc_mod

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sl = sc_mod.batched_scenes(num_scenes=12, nmin=2000, nmax=8000)
    mine = shard_scenes([sc.n for sc in sl], world)[rank]
    b = cb.DeviceBatch([sl[s] for s in mine], device="cuda:0")
    b.step(steps)
    full = b.state()
    res = {s: (b.scene_state(k, full)["x"], b.scene_state(k, full)["v"]) for k, s in enumerate(mine)}
    del b
    gathered = [None] * world
    dist.all_gather_object(gathered, res)
    if rank == 0:
        merged = {}
        for g in gathered:
            assert not set(g) & set(merged)
            merged.update(g)
        np.savez(os.path.join(out_dir, "engine_sharded.npz"),
                 **{f"x{k}": v[0] for k, v in merged.items()}, **{f"v{k}": v[1] for k, v in merged.items()})
    dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")
def test_engine_sharded_batch_equals_single_process(tmp_path):
    """Two processes (gloo) each step their shard of 12 batch scenes with the engine's batch solver
    for 60 substeps; gathered, every scene matches one process stepping all 12 together within the
    batch tolerance (positions 1e-4 of max(displacement, dx), velocities 1e-3 of their scale: the
    two runs sum grid nodes with float atomics in different orders)."""
    import crmpm_b200 as cb
    from gpu_helpers import rel_pos_err

    world, steps = 2, 60
    mp.start_processes(_engine_rank_main, args=(world, _free_port(), str(tmp_path), steps), nprocs=world,
                       start_method="spawn")
    got = np.load(tmp_path / "engine_sharded.npz")
    sl = scenes.batched_scenes(num_scenes=12, nmin=2000, nmax=8000)
    assert sorted(int(k[1:]) for k in got.files if k.startswith("x")) == list(range(len(sl)))
    cb.build_library()
    b = cb.DeviceBatch(sl)
    b.step(steps)
    full = b.state()
    for s, sc in enumerate(sl):
        ref = b.scene_state(s, full)
        assert rel_pos_err(got[f"x{s}"], ref["x"], sc.pos_mass[:, :3], sc.cell_size) <= 1e-4, s
        vscale = max(float(np.abs(ref["v"]).max()), 1e-3)
        assert float(np.abs(got[f"v{s}"] - ref["v"]).max()) <= 1e-3 * vscale + 1e-6, s
