#!/usr/bin/env python3
"""Throughput of the WCSPH step in particle-steps/s on B200.

Workload (default): the 1,048,576-particle tilting-box scene (preset
"large_tilting": r = 0.004, jitter +-0.2 r, N(0, 0.1) velocities, 2 x 1 x 1 m
box tilting 0 -> 15 deg about z over 1 s, fixed dt 5e-4). A step is one
FluidSimulator::update (sort, neighbourhood search, density, pressure,
non-pressure force, integrate + collision, CFL reduction) plus the box update
of that step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun as independent replicas (one scene per GPU, no
data-path collective; scaling "weak"); time is the max over ranks.
`--impl reference` times the reference's own CUDA kernels (compiled from its
sources into oracle/_ref by oracle/build_ref.py) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "fluid-simulation_b200"))

METRIC = "particle-steps/s"
# Algorithmic bytes per particle of each pass (compulsory reads + writes of
# the pass's own inputs/outputs, neighbour reads assumed cache-served).
PASS_BYTES = {
    "density_pass": 16 + 8,                       # pos -> rho, p
    "force_pass": 16 + 16 + 4 + 4 + 16 * 3,       # pos, vel, rho, p -> a_p, n, vlap
    "surface_integrate_pass": 16 * 6 + 4 + 16 * 3,  # pos, vel, n, rho, a_p, vlap -> a_np, pos, vel
    "keys_hist": 16 + 8,
    "radix_sort": 24,
    "reorder_cells": 4 + 32 + 32 + 8 + 4,
}
STEP_BYTES = 400  # algorithmic bytes per fluid particle-step of the reference step structure
# Algorithmic FP32 work per particle-step of the reference step structure:
# ~135 FLOP per neighbour pair over density, pressure force and non-pressure
# force (about 33 neighbours), plus ~9 FLOP per candidate distance test
# (about 216 candidates in 27 cells) in each of the three passes.
STEP_FLOP = 135 * 33 + 9 * 216 * 3
# Nominal FP32 (non-tensor) peak: 148 SMs x 128 FP32 lanes x 2 FLOP x 1.965 GHz.
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


BOX = {"large_tilting": "2x1x1 m tilting 0->15 deg/1 s", "dam_break": "1.0x0.6x0.6 m tank, walls on a 2r grid",
       "mesh_obstacle": "1 m cube, walls + level-4 icosphere R 0.15 on a 2r grid"}


def line_config(workload: str, n: int, delta: float, world: int, ms_per_step: float) -> dict:
    """The `config` block of a bench line (both arms use it)."""
    peak, peak_kind = measured_peaks()
    step_bw = STEP_BYTES * n / (ms_per_step * 1e-3) / 1e9
    return {"workload": workload, "particles": n, "dt": delta, "box": BOX.get(workload, "preset box"),
            "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (~250 MB resident per step)",
            "step_algorithmic_bytes_per_particle": STEP_BYTES,
            "step_hbm_fraction_of_" + peak_kind: step_bw / peak}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def _capture(workload: str, n: int):
    p = ROOT / "profiles" / f"dram_traffic_{workload}.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    return d if d.get("particles") == n else None


def measured_traffic(workload: str, n: int, kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu capture of this
    workload (profiles/dram_traffic_<workload>.json), or None."""
    d = _capture(workload, n)
    return None if d is None else d["bytes_per_launch"].get(kernel)


def measured_limits(workload: str, n: int, kernel: str):
    """Issue-active and L1TEX fractions of `kernel` from the same capture:
    what bounds a kernel whose HBM fraction is low."""
    d = _capture(workload, n)
    return None if d is None else d.get("utilisation", {}).get(kernel)


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) > 8:
                for k, name in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=None)
    return world, rank, local, dist


def max_over_ranks(value: float, dist, device) -> float:
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{device}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, device):
    if dist is not None:
        import torch

        dist.barrier(device_ids=[device])


def cpu_baseline(pre, budget_s: float = 15.0):
    """FP64 oracle (own C restatement) on the host cores, bounded sample."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    p, bx = pre.params, pre.box
    pos, vel = pre.pos.copy(), pre.vel.copy()
    bs, bm = (oracle.boundary_init(p, pre.bpos) if pre.bpos is not None else (None, None))
    steps = 0
    t0 = time.perf_counter()
    while True:
        r = oracle.step(p, bx, pos, vel, bs, bm, delta=pre.info.delta, nbr_cap=pos.shape[0] * 64)
        pos = r.pos.astype(np.float32)
        vel = r.vel.astype(np.float32)
        steps += 1
        el = time.perf_counter() - t0
        if el > budget_s or steps >= 50:
            break
    return {"value": pre.info.fluid_n * steps / el, "unit": METRIC, "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{steps} FP64 oracle steps of the same {pre.info.fluid_n}-particle workload, "
                      f"{el:.1f} s wall"}


def run_ours(args, world, rank, local, dist):
    import torch

    import wcsph

    torch.cuda.set_device(local)
    pre = wcsph.preset(args.workload, seed=args.seed)
    n = pre.info.fluid_n
    delta = pre.info.delta
    sim = pre.simulator(device=local)
    stream = torch.cuda.ExternalStream(sim.stream_handle(), device=f"cuda:{local}")
    boxes = [pre.box_at(k + 1) for k in range(args.warmup + args.steps + 8)] if pre.info.moving_box else None

    def one(k):
        if boxes is not None:
            sim.set_box(boxes[k])
        sim.step_n(1, delta)

    for k in range(args.warmup):
        one(k)
    sim.synchronize()
    barrier(dist, local)
    torch.cuda.synchronize(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for k in range(args.warmup, args.warmup + args.steps):
            one(k)
        e1.record(stream)
        e1.synchronize()
    sim.synchronize()
    torch.cuda.synchronize(local)
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, dist, local)
    barrier(dist, local)

    # per-pass device times (events between stages) for the roofline
    stages = {}
    for _ in range(5):
        for k, v in sim.kernel_timings().items():
            stages.setdefault(k, []).append(v)
    stage_ms = {k: statistics.median(v) for k, v in stages.items()}

    # end-to-end through the C ABI with host buffers: upload the state from
    # pinned host memory, per step upload the box and read back the metrics,
    # download the state at the end
    pin_pos = torch.from_numpy(pre.pos).pin_memory()
    pin_vel = torch.from_numpy(pre.vel).pin_memory()
    out_pos = torch.empty_like(pin_pos).pin_memory()
    out_vel = torch.empty_like(pin_vel).pin_memory()
    sim.synchronize()
    t0 = time.perf_counter()
    sim.set_state(pin_pos.numpy(), pin_vel.numpy())
    for k in range(args.steps):
        if boxes is not None:
            sim.set_box(boxes[k])
        sim.update(delta)
        sim.compute_state_metrics()
    sim.get_state(out=(out_pos.numpy(), out_vel.numpy()))   # straight into pinned memory
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist, local)
    box_bytes = 160
    h2d = (32 * n + args.steps * (box_bytes if boxes is not None else 0)) / args.steps
    d2h = (32 * n + 8 * args.steps) / args.steps

    launches = sim.launches_per_step() * args.steps
    sim.close()
    extras = {}
    if world == 1 and not args.no_extras:
        extras["batched"] = bench_batched(args)
        extras["rollout"] = bench_rollout()
        extras["mesh_obstacle"] = bench_mesh()
    if rank != 0:
        return None
    peak, peak_kind = measured_peaks()
    dom = max(("density_pass", "force_pass", "surface_integrate_pass"), key=lambda k: stage_ms.get(k, 0.0))
    traffic = measured_traffic(args.workload, n, dom)
    dom_ms = stage_ms[dom]
    achieved = PASS_BYTES[dom] * n / (dom_ms * 1e-3) / 1e9
    value = world * n * args.steps / (ms_max * 1e-3)
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded jittered lattice + N(0,0.1) velocities (preset large_tilting)",
        "config": line_config(args.workload, n, delta, world, ms_max / args.steps),
        "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"]},
        "e2e": {"value": world * n * args.steps / e2e_s, "unit": METRIC, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                     "ncu_utilisation": measured_limits(args.workload, n, dom),
                     "stage_ms": stage_ms,
                     "fp32": {"flop_per_particle_step": STEP_FLOP,
                              "achieved_tflops": STEP_FLOP * value / world / 1e12,   # per GPU
                              "peak_tflops": FP32_PEAK_TFLOPS, "peak_source": "nominal",
                              "frac": STEP_FLOP * value / world / 1e12 / FP32_PEAK_TFLOPS,
                              "dominant_kernel_fma_pipe": (measured_limits(args.workload, n, dom) or {}).get("fma_pipe")}},
    }
    line.update(extras)
    if not args.no_cpu_baseline:
        # timed on rank 0 of a single-GPU run only (a bounded host sample)
        line["cpu_baseline"] = cpu_baseline(pre, args.cpu_budget) if world == 1 else None
    return line


def bench_batched(args, n_scenes: int = 256, steps: int = 500):
    """Ensemble of 256 scenes (log-uniform 2048..65536 particles), the 500
    fixed steps of the workload: one persistent cooperative launch for all
    steps, the per-stage launches (one graph per step), and the same scenes
    stepped one after another through the single-scene path."""
    import wcsph

    pres, specs = ensemble_scenes(args, n_scenes)
    total = sum(p.info.fluid_n for p in pres)
    out = {"scenes": n_scenes, "particles": total, "steps": steps, "unit": METRIC}
    for mode, persistent in (("persistent", True), ("per_stage", False)):
        b = wcsph.BatchSimulator(pres[0].params, specs)
        b.set_persistent(persistent)
        b.step_n(3, 1e-3)
        ms = b.time_steps(steps, 1e-3)
        b.close()
        out[mode] = total * steps / (ms * 1e-3)
    sims = [s.simulator() for s in pres]
    for sim in sims:
        sim.step_n(3, 1e-3)
        sim.synchronize()
    t0 = time.perf_counter()
    for sim in sims:
        sim.step_n(steps, 1e-3)
        sim.synchronize()
    seq_s = time.perf_counter() - t0
    for sim in sims:
        sim.close()
    out["value"] = out["persistent"]
    out["sequential_value"] = total * steps / seq_s
    out["gain"] = out["value"] / out["sequential_value"]
    out["launches"] = {"persistent": 1, "per_stage": 14 * steps, "sequential": 14 * n_scenes * steps}
    return out


def ensemble_scenes(args, n_scenes: int = 256):
    import wcsph

    pres = [wcsph.preset_ensemble(args.seed + 1, k) for k in range(n_scenes)]
    specs = [wcsph.BatchSceneSpec(fluid_pos=s.pos, box=s.box, gravity=tuple(s.params.gravity),
                                  viscosity=s.params.viscosity, boundary_pos=s.bpos) for s in pres]
    return pres, specs


def ensemble_steps(args, k: int):
    """The batched ensemble's per-stage launches for 3 + k steps, untimed (a
    short, bounded workload for a launch-list capture)."""
    import wcsph

    pres, specs = ensemble_scenes(args)
    b = wcsph.BatchSimulator(pres[0].params, specs)
    b.set_persistent(False)
    b.step_n(3 + k, 1e-3)
    b.metrics()   # reads back, so the steps have finished
    b.close()


def bench_mesh(steps: int = 200, warmup: int = 10):
    """The mesh-obstacle scene (393,216 particles, walls and a sampled sphere,
    CFL-adaptive dt): device time per step over `steps` steps."""
    import torch

    import wcsph

    pre = wcsph.preset("mesh_obstacle")
    sim = pre.simulator()
    stream = torch.cuda.ExternalStream(sim.stream_handle())
    sim.step_n(warmup, pre.info.delta)
    sim.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step_n(steps, pre.info.delta)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    out = {"particles": pre.info.fluid_n, "boundary_particles": pre.info.boundary_n, "steps": steps,
           "ms_per_step": ms, "value": pre.info.fluid_n / (ms * 1e-3), "unit": METRIC, "last_dt": sim.last_dt()[0]}
    sim.close()
    return out


def bench_rollout():
    """Differentiable rollout (16,384 particles, 200 x 1e-3 steps, checkpoints
    every 20): backward time over forward time."""
    import wcsph

    pre = wcsph.preset("rollout_block")
    target = pre.pos.copy()
    target[:, 0] += 0.2
    target[:, 2] += 0.1
    sim = pre.simulator()
    sim.rollout_forward(20, 1e-3, 20, target)   # warm-up (allocations, module load)
    sim.rollout_backward()
    sim.set_state(pre.pos, pre.vel)
    sim.synchronize()
    t0 = time.perf_counter()
    loss = sim.rollout_forward(pre.info.steps, pre.info.delta, 20, target)
    t1 = time.perf_counter()
    sim.rollout_backward()
    t2 = time.perf_counter()
    sim.close()
    return {"particles": pre.info.fluid_n, "steps": pre.info.steps, "checkpoint_every": 20, "loss": loss,
            "forward_ms": (t1 - t0) * 1e3, "backward_ms": (t2 - t1) * 1e3, "backward_over_forward": (t2 - t1) / (t1 - t0)}


def run_reference(args, world, rank, local, dist):
    if rank != 0:
        return None
    sys.path.insert(0, str(ROOT / "oracle"))
    try:
        import refpath
    except Exception as e:  # noqa: BLE001
        return {"impl": "reference", "unavailable": f"reference harness not importable: {e}"}
    return refpath.bench_line(args, METRIC, lambda n, delta, ms: line_config(args.workload, n, delta, 1, ms))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large_tilting")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the ensemble and rollout measurements")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ensemble-only", type=int, default=0, metavar="K",
                    help="profiling entry: build the 256-scene ensemble, run 3 + K per-stage steps, print nothing")
    args = ap.parse_args()
    if args.ensemble_only:
        ensemble_steps(args, args.ensemble_only)
        return
    args.warmup = max(args.warmup, 3)
    world, rank, local, dist = dist_setup()
    try:
        if args.impl == "reference":
            line = run_reference(args, world, rank, local, dist)
        else:
            line = run_ours(args, world, rank, local, dist)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
