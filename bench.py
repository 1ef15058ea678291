"""Benchmark of the B200 MPM substep engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload slab|cube|pb|batch|adjoint|sdf]

Workload (default): the MLS-MPM tissue slab with a rigid probe -- 1.0 x 0.2 x 1.0 m slab, cell size
0.01 m, 8 particles per cell with seeded jitter (1,600,000 particles), Neo-Hookean E 2e4 / nu 0.4 /
density 1050, four side faces pinned by static box SDFs, a kinematic sphere SDF (r 0.05 m,
friction 0.3) pressing at 0.1 m/s, dt 1e-4.  One "step" is one MLS-MPM substep.  Inputs are
synthetic (seeded), the particle state (~350 MB) is larger than the 126 MB L2.

Our arm: `value` is particle-substeps/s with all data resident on the GPU (CUDA events on the
solver stream around K substeps replayed from a CUDA graph).  `e2e` drives the same substeps through
the C ABI's scene-style advance (CrB200SolverAdvance): 10 substeps per call, the probe pose uploaded
from pinned host memory before each call and the particle positions and velocities read back into
pinned host memory after it, as the reference's Scene::advance does.

Reference arm (--impl reference): the reference's own CPU solver arithmetic (oracle/_ref, built
from the reference's headers) on the same workload, single-threaded as the reference's CPU solver
is.  On more than one GPU, rank 0 alone runs it.

Batched workload (--workload batch): 256 independent MLS-MPM scenes, each a 64^3-cell grid of
0.02 m with one elastic box of seeded size (2k-64k particles, log-uniform), a ground plane and a
sphere SDF, dt 2e-4.  `value` is the aggregate particle-substeps/s of one batch solver stepping all
scenes together (one launch per phase, CUDA graph); `one_by_one` is the same scenes run one after
another on the plain single-scene solver (one solver per scene, a shared stream, CUDA graphs).

SDF workload (--workload sdf): the GPU triangle-mesh SDF builder (CrB200SdfCompute, the work of
the reference's SdfBuilder::computeSdf + computeSdfGradient) on a 5120-triangle sphere mesh
(radius 0.3 m) over a 0.005 m grid (129^3 = 2.15M nodes).  One "step" is one build.  `value` is
nodes/s of the two kernels (CUDA events inside the library around them); `e2e` is nodes/s of the
whole call from host mesh arrays plus the copy of the grid into pinned host memory.  The CPU
baseline and the reference arm run the reference's own SdfBuilder (oracle/_ref/libref_sdf.so,
compiled from its sources) on the same mesh over a coarser grid.

Multi-GPU: one scene does not shard; N GPUs run N independent replicas (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cressim-mpm_b200"))

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, period_ms: int = 100):
        self.gpu = gpu_index
        self.period = period_ms
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", f"-lms={self.period}"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


METRICS = {
    "slab": "particle-substeps/s (MLS-MPM 1.6M p)",
    "cube": "particle-substeps/s (MLS-MPM 4096-particle cube)",
    "pb": "particle-steps/s (PB-MPM cutting, 540k p, 20 iterations per step)",
    "sdf": "SDF grid nodes/s (triangle-mesh SDF build, 5120-triangle sphere, 129^3 nodes)",
}
UNITS = {"slab": "particle-substeps/s", "cube": "particle-substeps/s", "pb": "particle-steps/s", "sdf": "nodes/s"}

SDF_MESH = dict(radius=0.3, subdivisions=4, cell=0.005, fatten=0.02)


def sdf_mesh():
    from crmpm_b200 import meshes

    return meshes.icosphere(SDF_MESH["radius"], SDF_MESH["subdivisions"])


def sdf_reference_run(cell: float, steps: int, budget_s: float):
    """The reference's SdfBuilder (oracle/_ref/libref_sdf.so) on the benchmark mesh over a grid of
    spacing `cell`: (nodes/s, builds timed, seconds, nodes per build) or None."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as op

    if not op.ref_sdf_available():
        return None
    P, T = sdf_mesh()
    t0 = time.perf_counter()
    done = nodes = 0
    while done < steps:
        dims, _, _ = op.ref_sdf(P, T, cell, SDF_MESH["fatten"])
        nodes = int(np.prod(dims))
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return nodes * done / el, done, el, nodes


def run_sdf(args, rank, world, local):
    """GPU triangle-mesh SDF build (CrB200SdfCompute) on the benchmark mesh."""
    import torch

    import crmpm_b200 as cb

    cb.build_library()
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    P, T = sdf_mesh()
    cell, fatten = SDF_MESH["cell"], SDF_MESH["fatten"]
    d = cb.sdf_desc(P, T, cell, fatten)
    dims = tuple(int(v) for v in d.sdfDimension)
    n = int(np.prod(dims))
    stream = torch.cuda.Stream(device=dev)
    out = torch.empty((n, 4), dtype=torch.float32, device=dev)
    host = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
    for _ in range(args.warmup):
        cb.build_sdf(P, T, cell, fatten, out=out, stream=stream.cuda_stream)
    torch.cuda.synchronize(dev)

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize(dev)
    launches0 = cb.kernel_launch_count()
    k_nodes = k_grad = 0.0
    for _ in range(args.steps):
        cb.build_sdf(P, T, cell, fatten, out=out, stream=stream.cuda_stream)
        a, b = cb.sdf_last_kernel_ms()
        k_nodes += a
        k_grad += b
    torch.cuda.synchronize(dev)
    barrier(world)
    launches = cb.kernel_launch_count() - launches0
    clocks = sampler.stop()
    ms = max_over_ranks(k_nodes + k_grad, world)
    value = world * n * args.steps / (ms / 1e3)

    # end to end: host mesh arrays in, grid out into pinned host memory, CUDA events on the stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for _ in range(args.steps):
        cb.build_sdf(P, T, cell, fatten, out=out, stream=stream.cuda_stream)
        with torch.cuda.stream(stream):
            host.copy_(out, non_blocking=True)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
    leaves = -(-len(T) // 8)
    p2 = 1 << max(0, (leaves - 1).bit_length())
    h2d = 16 * (3 * 8 * p2 + 4 * 2 * p2)  # triangle records + tree nodes the library uploads
    peak, peak_kind = hbm_peak()
    grad_bytes = 20.0 * n  # read one distance, write one float4 per node (neighbours from cache)
    grad_gbs = grad_bytes * args.steps / (k_grad / 1e3) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = sdf_reference_run(0.02, steps=3, budget_s=20.0)
        if r is not None:
            v, done, el, nodes = r
            cpu = {"value": v, "unit": "nodes/s", "cores": 1, "kind": "reference",
                   "sample": f"{done} build(s) of the same mesh over a 0.02 m grid ({nodes} nodes, {el:.1f} s) by "
                             f"the reference's SdfBuilder compiled from its sources"}
    out_line = {
        "metric": METRICS["sdf"],
        "value": value,
        "unit": "nodes/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (procedural icosphere mesh)",
        "config": {"workload": f"triangle-mesh SDF build: icosphere r 0.3 m, {len(T)} triangles, cell {cell} m, fatten "
                               f"{fatten} m, grid {dims[0]}x{dims[1]}x{dims[2]} ({n} nodes), normalised gradient",
                   "parallelism": f"replicas x{world}", "l2": "output grid 34 MB written once per build"},
        "roofline": {"bound": "alu", "kernel": "k_sdfNodes", "achieved": None, "peak": None, "unit": None,
                     "frac": None, "traffic": None,
                     "note": "tree walk bound by FP32/MUFU issue (closest point, solid angles); the HBM-bound "
                             "gradient kernel is reported under gradient_kernel",
                     "kernel_ms": {"k_sdfNodes": k_nodes / args.steps, "k_sdfGradient": k_grad / args.steps},
                     "gradient_kernel": {"bound": "hbm", "achieved": grad_gbs, "peak": peak, "unit": "GB/s",
                                         "frac": grad_gbs / peak, "peak_source": peak_kind}},
        "e2e": {"value": world * n * args.steps / (e2e_ms / 1e3), "unit": "nodes/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 16 * n},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if cpu is not None:
        out_line["cpu_baseline"] = cpu
    return out_line


def make_workload(name):
    from crmpm_b200 import scenes

    if name == "slab":
        return scenes.tissue_slab(), "MLS-MPM tissue slab + rigid probe, 1.6M particles, 121x61x121 grid, dt 1e-4"
    if name == "cube":
        return scenes.cube_drop(), "MLS-MPM elastic cube drop, 4096 particles, 41^3 grid, dt 2e-4"
    if name == "pb":
        sc = scenes.pb_cutting()
        return sc, (f"PB-MPM slab cut by a kinematic quad-slicer blade, {sc.n} particles, 101x51x101 grid, dt 2e-3, "
                    f"{sc.iterations} solver iterations per step")
    raise SystemExit(f"unknown workload {name}")


def cpu_reference_run(scene, steps: int, warmup: int, budget_s: float):
    """The reference's CPU solver (oracle/_ref) on the workload: (substeps/s * particles, timed, note)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as op

    if not op.ref_available():
        return None, 0, "oracle/_ref not built"
    r = op.RefOracle(scene)
    r.compute_initial_data()
    for _ in range(warmup):
        r.step(1)
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        r.step(1)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return scene.n * done / el, done, el


def snapshot_state(ds):
    """Device copies of a scene's particle state (x, v, F, C, V0) and shape poses."""
    import torch

    n = ds.scene.n
    ds.sync()
    F = torch.empty((n, 9), dtype=torch.float32, device=ds.device)
    Cm = torch.empty_like(F)
    V0 = torch.empty(n, dtype=torch.float32, device=ds.device)
    ds.solver.copy_particle_state(n, F.data_ptr(), Cm.data_ptr(), V0.data_ptr())
    ds.sync()
    return ds.pos.clone(), ds.vel.clone(), F, Cm, V0, ds.sh["position"].clone()


def restore_state(ds, snap):
    """Put a snapshot_state back (SetParticleState also drops the carried P2G records)."""
    import torch

    pos, vel, F, Cm, V0, shp = snap
    ds.sync()
    ds.pos.copy_(pos)
    ds.vel.copy_(vel)
    ds.sh["position"].copy_(shp)
    torch.cuda.synchronize(ds.device)
    ds.solver.set_particle_state(ds.scene.n, F.data_ptr(), Cm.data_ptr(), V0.data_ptr())
    ds.sync()


def run_ours(args, rank, world, local):
    import torch

    import crmpm_b200 as cb

    cb.build_library()
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    from crmpm_b200 import scenes as scenes_mod

    scene, desc = make_workload(args.workload)
    n = scene.n
    ds = cb.DeviceScene(scene, device=dev, compute_initial=not args.deterministic)
    if args.deterministic:  # the whole run in deterministic mode (CRB200_OPT_DETERMINISTIC)
        ds.solver.set_option(cb.OPT_DETERMINISTIC, 1)
        ds.compute_initial_data()
    s = ds.solver
    stream = ds.stream
    if args.resident:
        s.set_option(cb.OPT_RESIDENT, 1)
    # warm-up (graph capture happens on the first replay), then the launch-shape autotuner
    ds.step(max(args.warmup, 3))
    tuned = (0, 0, 0) if args.quick else s.autotune(10)  # --quick: short runs for profiler launch lists
    ds.step(3)
    ds.sync()
    st = s.grid_stats()
    touched_nodes = st["touched_nodes"]
    # the state the timed region starts from: the end-to-end pass below restarts from it, so that
    # both measure the same substeps of the simulation
    snap = None if args.quick else snapshot_state(ds)

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize(dev)
    launches0 = cb.kernel_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.step_many(args.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    barrier(world)
    launches = cb.kernel_launch_count() - launches0
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world)
    value = world * n * args.steps / (ms_max / 1e3)
    if args.quick:
        return {"metric": METRICS[args.workload] + (" deterministic" if args.deterministic else ""), "value": value,
                "unit": UNITS[args.workload],
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "quick": True, "gpu_launches": int(launches)}

    # per-kernel timing pass (CUDA events around each phase on the solver stream)
    s.set_option(cb.OPT_PHASE_TIMING, 1)
    s.phase_times(reset=True)
    s.resident_kernel_time(reset=True)
    nprof = min(50, max(10, args.steps // 10))
    s.step_many(nprof)  # one call, as in the timed region
    phase_ms, nph = s.phase_times(reset=True)
    fused_ms, fused_n = s.resident_kernel_time(reset=True)
    s.set_option(cb.OPT_PHASE_TIMING, 0)
    per_phase = {name: phase_ms[i] / max(nph, 1) for i, name in enumerate(cb.PHASES)}
    peak, peak_kind = hbm_peak()
    # algorithmic bytes (200 B per particle and 64 B per touched node per substep) split by kernel:
    # the fused kernel does one substep's G2P and the next one's P2G, so it reads and writes the
    # particle state once (200 B) and reads one grid and writes the next (32 B per node)
    alg = {"p2g": 104.0 * n + 16.0 * touched_nodes, "g2p": 96.0 * n + 16.0 * touched_nodes,
           "grid_update": 32.0 * touched_nodes, "g2p2g": 200.0 * n + 32.0 * touched_nodes}
    if fused_n > 0:
        # the resident path: the fused G2P -> P2G kernel, timed per launch
        dom = "g2p2g"
        per_phase["g2p2g_per_launch"] = fused_ms / fused_n
        achieved = alg[dom] / (fused_ms / fused_n / 1e3) / 1e9
    else:
        dom = max(("p2g", "g2p", "grid_update"), key=lambda k: per_phase[k])
        achieved = alg[dom] / (per_phase[dom] / 1e3) / 1e9
    substep_bytes = 200.0 * n + 64.0 * touched_nodes
    if scene.solver_type == scenes_mod.SOLVER_PB:
        # PB-MPM step: per iteration read x, v, F, m and read / write C (136 B / particle) and 64 B per
        # touched node, plus the integration's 200 B / particle; the phases fold the iterations
        # together, so the roofline is given for the whole step
        substep_bytes = scene.iterations * (136.0 * n + 64.0 * touched_nodes) + 200.0 * n
        dom = "step"
        achieved = substep_bytes / (ms / 1e3 / args.steps) / 1e9
    substep_gbs = substep_bytes / (ms / 1e3 / args.steps) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    if os.path.exists(tfile):
        with open(tfile) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 3 and not line.startswith("#") and parts[:2] == [args.workload, dom]:
                    traffic = float(parts[2])

    # end to end through the C ABI: scene-style advance with host buffers, pipelined as the
    # reference's Scene::advance / fetchResults pair allows (CrB200SolverAdvanceAsync): frame k+1's
    # substeps run while frame k's positions and velocities are copied into pinned host memory
    restore_state(ds, snap)
    frame_substeps = 10
    frame_dt = float(np.float32(scene.dt) * frame_substeps) * 0.999
    host_pos = [torch.empty((ds.num_max, 4), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    host_vel = [torch.empty((ds.num_max, 4), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    probe = scene.shapes.shape_ids[-1]  # the moving shape (probe or blade), moved along its velocity
    pose0 = ds.sh["position"][probe].cpu()
    probe_vel = scene.shapes.lin_vel[probe, :3].astype(np.float64)
    frames = max(20, args.steps // frame_substeps)
    # one pinned pose per frame: a frame's upload may still be queued when the next is written
    poses = [torch.empty(4, dtype=torch.float32, pin_memory=True) for _ in range(frames)]
    for f_ in range(frames):
        poses[f_].copy_(pose0)
        poses[f_][:3] += torch.tensor(probe_vel * scene.dt * frame_substeps * (f_ + 1), dtype=torch.float32)
    s.advance(frame_dt, host_pos[0].data_ptr(), host_vel[0].data_ptr())  # warm-up
    s.advance_async(frame_dt, host_pos[1].data_ptr(), host_vel[1].data_ptr())
    s.fetch_results()
    barrier(world)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    sub_total = 0
    for f_ in range(frames):
        with torch.cuda.stream(stream):
            ds.sh["position"][probe].copy_(poses[f_], non_blocking=True)
        b = f_ & 1  # two buffer pairs: copies into one buffer happen in call order
        sub_total += s.advance_async(frame_dt, host_pos[b].data_ptr(), host_vel[b].data_ptr())
    s.fetch_results()
    torch.cuda.synchronize(dev)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = world * n * sub_total / e2e_s
    h2d = 16 * frames
    d2h = 32 * n * frames

    # the same substeps in deterministic mode (CRB200_OPT_DETERMINISTIC: bit-reproducible runs)
    dd = cb.DeviceScene(scene, device=dev, compute_initial=False)
    dd.solver.set_option(cb.OPT_DETERMINISTIC, 1)
    dd.compute_initial_data()
    dd.step(max(args.warmup, 3))
    dd.sync()
    d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dsteps = min(args.steps, 500)
    d0.record(dd.stream)
    dd.solver.step_many(dsteps)
    d1.record(dd.stream)
    d1.synchronize()
    dms = d0.elapsed_time(d1) / dsteps
    det = {"ms_per_step": dms, "value": n / (dms / 1e3), "steps": dsteps,
           "note": "CRB200_OPT_DETERMINISTIC: P2G block tiles summed in a fixed order, cells in id order, "
                   "coupling reduced in a fixed order; two runs from the same state agree bit for bit"}
    del dd

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, done, el = cpu_reference_run(scene, steps=20, warmup=1, budget_s=25.0)
        if v is not None:
            cpu = {"value": v, "unit": "particle-substeps/s", "cores": 1, "kind": "reference",
                   "sample": f"{done} substeps of the same workload ({scene.n} particles, {el:.1f} s) with the reference's "
                             f"serial CPU solver arithmetic built from its own headers"}
    status = s.status()
    extras = None
    if args.workload == "slab" and world == 1 and not args.no_extras:
        del ds
        torch.cuda.synchronize(dev)
        extras = bench_extras(args, local, scene, value)
    out = {
        "metric": METRICS[args.workload] + (" deterministic" if args.deterministic else ""),
        "value": value,
        "unit": UNITS[args.workload],
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded jittered particles)",
        "config": {"workload": desc, "particles": n, "grid": list(s.grid_dims()), "dt": scene.dt,
                   "substeps_per_step": 1, "parallelism": f"replicas x{world}",
                   "path": "resident cell-ordered (CRB200_OPT_RESIDENT)" if args.resident else "particle-id order",
                   "l2": "inputs larger than L2 (particle state ~350 MB)", "touched_nodes": touched_nodes,
                   "autotuned_launch": {"update_ctas_per_sm": tuned[0], "accumulate_x": tuned[1], "sort_x": tuned[2]}},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "phase_ms": per_phase, "substep_gbs_algorithmic": substep_gbs,
                     "substep_frac": substep_gbs / peak},
        "e2e": {"value": e2e_value, "unit": "particle-substeps/s", "h2d_bytes_per_step": h2d // frames,
                "d2h_bytes_per_step": d2h // frames, "substeps_per_step": frame_substeps},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "status": status,
    }
    if det is not None:
        out["deterministic"] = det
    if cpu is not None:
        out["cpu_baseline"] = cpu
    if extras is not None:
        out.update(extras)
    return out


def bench_extras(args, local, slab_scene, slab_value):
    """The engine's other targets, each timed outside the headline's timed region with CUDA events
    on its own stream and bounded to a few seconds of GPU work, so that a default run reports them:

    * reference_gpu: the reference's own CUDA solver on the slab over 200 substeps (the >= 3x bar);
    * batch: the 256-scene batch against the same scenes one by one on the plain solver (>= 2x);
    * adjoint: backward over plain forward for the 64k cube and a 64-scene batch of it (<= 3x);
    * pb: the PB-MPM cutting workload against the reference's CUDA solver on the same scene.
    A part that fails reports its error instead of stopping the run."""
    import torch

    import crmpm_b200 as cb
    from crmpm_b200 import scenes

    dev = f"cuda:{local}"
    out = {}

    def guard(name, fn):
        try:
            out[name] = fn()
        except Exception as e:  # noqa: BLE001 - reported in the line, the headline stands
            out[name] = {"error": f"{type(e).__name__}: {str(e).splitlines()[0][:200] if str(e) else ''}"}
        torch.cuda.synchronize(dev)

    def ref_slab():
        r = reference_gpu_run(slab_scene, args, steps=200)
        if r is not None and "value" in r:
            r["engine_over_reference"] = slab_value / r["value"]
        return r

    def batch():
        r = batch_measure(20, 3, 0, 1, local)
        return {"value": r["value"], "unit": "particle-substeps/s", "substeps": 20, "scenes": len(r["sl"]),
                "particles": r["n"], "one_by_one": r["one_value"], "one_by_one_substeps": r["k1"],
                "batch_over_one_by_one": r["value"] / r["one_value"],
                "how": "one batch solver (one launch per phase, CUDA graph) vs one plain solver per scene on a "
                       "shared stream (CUDA graph per scene)"}

    def adjoint():
        T, single, b64 = adjoint_measure(local)
        return {"workload": ADJOINT_CONFIG, "substeps": T, "single": single, "batch64": b64,
                "target": "backward <= 3x the plain forward"}

    def pb():
        sc = scenes.pb_cutting()
        ds = cb.DeviceScene(sc, device=dev)
        ds.step(3)
        ds.sync()
        steps = 20
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ds.stream)
        ds.solver.step_many(steps)
        e1.record(ds.stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        del ds
        r = {"value": sc.n / (ms / 1e3), "unit": "particle-steps/s", "ms_per_step": ms, "steps": steps,
             "particles": sc.n, "iterations": sc.iterations}
        ref = reference_gpu_run(sc, args, steps=steps)
        if ref is not None:
            r["reference_gpu"] = ref
            if "value" in ref:
                r["engine_over_reference"] = r["value"] / ref["value"]
        return r

    guard("reference_gpu", ref_slab)
    guard("batch", batch)
    guard("adjoint", adjoint)
    guard("pb", pb)
    return out


def batch_measure(steps, warmup, rank, world, local, sampler=None):
    """256 batched scenes (this rank's shard) stepped by one batch solver, then the same scenes one
    by one on plain single-scene solvers; CUDA events on each stream, max over ranks."""
    import torch

    import crmpm_b200 as cb
    from crmpm_b200 import scenes
    from crmpm_b200.sharding import shard_scenes

    dev = f"cuda:{local}"
    sl_all = scenes.batched_scenes()
    # N GPUs: each rank steps its own scenes (largest-first balance), no data-path collective
    mine = shard_scenes([sc.n for sc in sl_all], world)[rank]
    sl = [sl_all[k] for k in mine]
    n = sum(sc.n for sc in sl_all)
    b = cb.DeviceBatch(sl, device=dev)
    b.step(max(warmup, 3))
    tuned = b.solver.autotune(4)
    b.step(2)
    b.sync()
    touched_nodes = b.solver.grid_stats()["touched_nodes"]

    def timed(stream, fn):
        barrier(world)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), world)

    if sampler is not None:
        sampler.start()
        time.sleep(0.3)
    launches0 = cb.kernel_launch_count()
    ms = timed(b.stream, lambda: b.solver.step_many(steps))
    launches = cb.kernel_launch_count() - launches0
    clocks = sampler.stop() if sampler is not None else None
    value = n * steps / (ms / 1e3)
    status = b.solver.status()
    del b

    # one by one: a plain solver per scene, all on one stream, each scene's substeps in turn
    shared = torch.cuda.Stream(device=dev)
    singles = [cb.DeviceScene(sc, device=dev, stream=shared) for sc in sl]
    for g in singles:
        g.step(3)
    k1 = min(steps, 50)
    ms1 = timed(shared, lambda: [g.solver.step_many(k1) for g in singles])
    one_value = n * k1 / (ms1 / 1e3)
    del singles
    peak, peak_kind = hbm_peak()
    n_mine = sum(sc.n for sc in sl)
    substep_gbs = (200.0 * n_mine + 64.0 * touched_nodes) / (ms / 1e3 / steps) / 1e9
    return dict(n=n, sl=sl, ms=ms, value=value, one_value=one_value, k1=k1, tuned=tuned, launches=launches,
                clocks=clocks, touched_nodes=touched_nodes, substep_gbs=substep_gbs, peak=peak, peak_kind=peak_kind,
                status=status)


def run_batch(args, rank, world, local):
    """256 batched scenes vs the same scenes one by one on the plain solver."""
    import torch

    import crmpm_b200 as cb

    cb.build_library()
    torch.cuda.set_device(local)
    r = batch_measure(args.steps, args.warmup, rank, world, local, sampler=ClockSampler(local))
    n, sl, ms, value, one_value, k1 = r["n"], r["sl"], r["ms"], r["value"], r["one_value"], r["k1"]
    tuned, launches, clocks, touched_nodes = r["tuned"], r["launches"], r["clocks"], r["touched_nodes"]
    substep_gbs, peak, peak_kind = r["substep_gbs"], r["peak"], r["peak_kind"]
    return {
        "metric": "particle-substeps/s (batched MLS-MPM, 256 scenes)",
        "value": value,
        "unit": "particle-substeps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded jittered particles)",
        "config": {"workload": "256 MLS-MPM scenes, 64^3-cell grids of 0.02 m, 2k-64k particles each (log-uniform), "
                               "plane + sphere SDF per scene, dt 2e-4", "particles": n, "scenes": len(sl),
                   "touched_nodes_rank0": touched_nodes, "l2": "inputs larger than L2 (particle state ~1 GB)",
                   "parallelism": f"scene shards x{world}", "scenes_rank0": len(sl),
                   "autotuned_launch": {"update_ctas_per_sm": tuned[0], "accumulate_x": tuned[1], "sort_x": tuned[2]}},
        "one_by_one": {"value": one_value, "unit": "particle-substeps/s", "substeps": k1,
                       "how": "one plain solver per scene, shared stream, CUDA graph per scene"},
        "batch_over_one_by_one": value / one_value,
        "roofline": {"bound": "hbm", "kernel": "substep", "substep_gbs_algorithmic": substep_gbs, "peak": peak,
                     "unit": "GB/s", "frac": substep_gbs / peak, "peak_source": peak_kind},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "status": r["status"],
    }


ADJOINT_CONFIG = ("64k-particle Neo-Hookean cube (0.4 m, dx 0.02, 8 ppc) 1 cm above a ground plane at -1 m/s, 200 "
                  "substeps of 2e-4 s, positions captured at 50/100/150/200, checkpoint every 20; gradients at E 8e3, "
                  "nu 0.25 against targets made at E 2e4, nu 0.35")


def adjoint_measure(local, quick=False, with_batch=True):
    """Forward record + backward of the material-identification cube (and of a 64-scene batch of
    it), each against the plain forward of the same substeps; CUDA events on the solver stream."""
    import torch

    import crmpm_b200 as cb
    from crmpm_b200 import scenes
    from crmpm_b200.adjoint import Trajectory, lame

    dev = f"cuda:{local}"
    T, caps, K = 200, (50, 100, 150, 200), 20
    if quick:  # short run for profiler launch lists: 40 substeps, the single cube only
        T, caps, K = 40, (20, 40), 20

    def cube(seed):
        return scenes.material_cube(seed=seed, E=8e3, nu=0.25, drop=0.01, v0=(0.0, -1.0, 0.0))

    def measure(ds, sl):
        n = ds.scene.n
        run = Trajectory(ds, T, caps, K)
        s = ds.stream

        def params(E, nu):
            lam, mu = lame(E, nu)
            return (torch.full((n,), lam, device=dev), torch.full((n,), mu, device=dev),
                    torch.tensor(ds.scene.vel[:, :3], device=dev))

        target = run.forward(*params(2e4, 0.35))
        guess = params(8e3, 0.25)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        for rep in range(2):  # the first pass allocates the tape
            torch.cuda.synchronize(dev)
            ev[0].record(s)
            pos = run.forward(*guess)
            ev[1].record(s)
            g = 2.0 * (pos - target) / (3 * n)
            torch.cuda.synchronize(dev)
            ev[2].record(s)
            gl, gm, gv = run.backward(g)
            ev[3].record(s)
            torch.cuda.synchronize(dev)
        # plain forward of the same substeps (graph replay)
        ev[4].record(s)
        ds.solver.step_many(T)
        ev[5].record(s)
        ev[5].synchronize()
        fwd_rec, bwd, plain = ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3]), ev[4].elapsed_time(ev[5])
        return dict(particles=n, record_ms=fwd_rec, backward_ms=bwd, plain_forward_ms=plain,
                    backward_over_plain_forward=bwd / plain, grad_E_sign_check=float(gl.sum()))

    single = measure(cb.DeviceScene(cube(1005), device=dev), None)
    batch = None
    if with_batch and not quick:
        batch = measure(cb.DeviceBatch([cube(2000 + s) for s in range(64)], device=dev), None)
    return T, single, batch


def run_adjoint(args, rank, world, local):
    """Material identification: forward record + adjoint of the 64k-particle cube (and a 64-scene batch)."""
    import torch

    import crmpm_b200 as cb

    cb.build_library()
    torch.cuda.set_device(local)
    T, single, batch = adjoint_measure(local, quick=args.quick)
    n = single["particles"]
    value = n * T / (single["backward_ms"] / 1e3)
    return {
        "metric": "particle-substeps/s (adjoint MLS-MPM, 64k-particle cube)",
        "value": value,
        "unit": "particle-substeps/s",
        "n_gpus": world,
        "steps": T,
        "warmup": 1,
        "ms_per_step": single["backward_ms"] / T,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded jittered particles)",
        "config": {"workload": ADJOINT_CONFIG},
        "single": single,
        "batch64": batch,
    }


def run_reference(args, rank, world):
    if rank != 0:
        return None
    if args.workload == "sdf":
        r = sdf_reference_run(0.04, steps=args.steps, budget_s=120.0)
        if r is None:
            return {"impl": "reference", "unavailable": "reference SDF builder (oracle/_ref/libref_sdf.so) is not built"}
        v, done, el, nodes = r
        return {"impl": "reference", "metric": METRICS["sdf"], "value": v, "unit": "nodes/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / max(done, 1) * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (procedural icosphere mesh)",
                "config": {"workload": "the benchmark's 5120-triangle sphere over a 0.04 m grid (a bounded sample)"},
                "cpu_baseline": {"value": v, "unit": "nodes/s", "cores": 1, "kind": "reference",
                                 "sample": f"{done} builds of {nodes} nodes ({el:.1f} s), reference SdfBuilder"},
                "e2e": {"value": v, "unit": "nodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    scene, desc = make_workload(args.workload)
    v, done, el = cpu_reference_run(scene, steps=args.steps, warmup=min(args.warmup, 3), budget_s=150.0)
    if v is None:
        return {"impl": "reference", "unavailable": "reference CPU solver driver (oracle/_ref) is not built"}
    sample = (f"{done} of {args.steps} requested steps of the workload ({scene.n} particles) timed ({el:.1f} s), "
              f"reference serial CPU solver arithmetic built from its own headers")
    gpu = reference_gpu_run(scene, args)
    line = {
        "impl": "reference",
        "metric": METRICS[args.workload],
        "value": v,
        "unit": UNITS[args.workload],
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": el / max(done, 1) * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded jittered particles)",
        "config": {"workload": desc, "particles": scene.n, "substeps_per_step": 1},
        "cpu_baseline": {"value": v, "unit": UNITS[args.workload], "cores": 1, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": UNITS[args.workload], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if gpu is not None:
        line["reference_gpu"] = gpu
    return line


def reference_gpu_run(scene, args, steps=None):
    """The reference's own CUDA solver (oracle/_ref/ref_gpu_driver: src/solver/gpu_*_mpm_solver.cu
    built for sm_100a) on the same workload, timed with CUDA events on its stream after warm-up
    substeps, inputs resident in HBM.  None when the driver is not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as op

    if not op.ref_gpu_available():
        return None
    if steps is None:
        steps = min(max(args.steps, 200), 500 if scene.solver_type != 3 else 100)
    try:
        r = op.ref_gpu_run(scene, steps, warmup=max(args.warmup, 3))
    except (RuntimeError, OSError, subprocess.TimeoutExpired) as e:
        return {"unavailable": str(e).splitlines()[0][:200]}
    ms = r["ms_per_substep"]
    return {"value": scene.n / (ms / 1e3), "unit": UNITS[args.workload], "ms_per_step": ms, "steps": steps,
            "warmup": max(args.warmup, 3),
            "note": "the reference's GpuMlsMpmSolver / GpuPbMpmSolver / GpuStandardMpmSolver compiled from its own "
                    "sources for sm_100a (-O3), driven through its MpmSolver interface; CUDA events around the "
                    "timed substeps"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="slab", choices=["slab", "cube", "pb", "batch", "adjoint", "sdf"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--deterministic", action="store_true",
                    help="single-scene workloads: run the timed substeps with CRB200_OPT_DETERMINISTIC on")
    ap.add_argument("--resident", action="store_true",
                    help="single-scene MLS workloads: the resident cell-ordered path (CRB200_OPT_RESIDENT)")
    ap.add_argument("--quick", action="store_true",
                    help="timed region only (no phase pass, e2e or CPU baseline): for profiler launch lists")
    ap.add_argument("--no-extras", action="store_true",
                    help="slab workload: skip the batch / adjoint / PB / reference-GPU figures after the headline")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    rank, world, local = dist_setup(args.gpus)
    if args.workload == "batch":
        out = run_batch(args, rank, world, local)
    elif args.workload == "adjoint":
        out = run_adjoint(args, rank, world, local)
    elif args.workload == "sdf":
        out = run_sdf(args, rank, world, local)
    else:
        out = run_ours(args, rank, world, local)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
