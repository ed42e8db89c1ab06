"""Batched many-scene stepping: throughput and per-scene latency.

Workload: 256 independent 2-D channels (solver constants of the small
channel: r = 0.01, h = 0.04, dt = 4e-4, M = N/16 inverse-CDF samples),
fluid counts log-uniform in [2k, 60k], inflow U(0.5, 2), cylinder radius
U(0.05, 0.15); seeded, synthetic.

Arms:
  * batch: one context, every scene advanced by dv_batch_step; the steps are
    captured in a CUDA graph (2 steps) and replayed.  The far-field tile
    (targets per thread) is chosen by timing graph replays of each candidate.
  * one at a time: each scene on its own single-scene context, stepped by
    KarmanVortexSolver.step() in a loop over the scenes.

Reports aggregate fluid particle-steps/s of both arms and the per-scene step
latency p50 / p99 (batch: the batch step time, which is the latency of every
scene in it; one at a time: each scene's own step time).  Times are CUDA-event
device times.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from .batch import SceneBatch, channel_batch_configs


def _ev_time(fn, reps):
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run(n_scenes: int = 256, seed: int = 0, warmup: int = 4, reps: int = 10, lone_rounds: int = 3,
        tiles=(2, 4, 6, 8)) -> dict:
    cfgs, Ns = channel_batch_configs(n_scenes=n_scenes, seed=seed)
    t0 = time.perf_counter()
    b = SceneBatch(cfgs)
    out = {"workload": f"{n_scenes} 2-D channels, fluid log-uniform [2k, 60k], r 0.01, M = N/16",
           "n_scenes": n_scenes, "build_seconds": time.perf_counter() - t0}
    for _ in range(warmup):
        b.step()
    torch.cuda.synchronize()
    out["eager_step_ms"] = _ev_time(b.step, 2)
    # autotune the far-field tile on graph replays of the real state
    tune = {}
    for tt in tiles:
        b._check(b.lib.dv_set_far_tile(b.ctx, int(tt)), "dv_set_far_tile")
        b.capture(2)
        b.replay()
        tune[tt] = _ev_time(b.replay, 2) / 2
    best = min(tune, key=tune.get)
    b._check(b.lib.dv_set_far_tile(b.ctx, int(best)), "dv_set_far_tile")
    b.capture(2)
    b.replay()
    st = b.states()
    n_fluid = sum(s["n_fluid"] for s in st)
    n_all = sum(s["end"] - s["start"] for s in st)
    ms = _ev_time(b.replay, reps) / 2
    st2 = b.states()
    eager_same_state = _ev_time(b.step, 2)  # eager steps from the state the graph timing ended in
    out["batch"] = {"ms_per_step": ms, "particle_steps_per_s": n_fluid / (ms * 1e-3),
                    "fluid_particles": n_fluid, "all_particles": n_all,
                    "latency_ms_p50": ms, "latency_ms_p99": ms, "far_tile_targets_per_thread": best,
                    "tile_sweep_ms": {str(k): v for k, v in tune.items()},
                    "iters_div_max": max(s["iters_div"] for s in st2),
                    "iters_p_max": max(s["iters_p"] for s in st2),
                    "iters_p_mean": float(np.mean([s["iters_p"] for s in st2])),
                    "scenes_ever_at_iteration_cap": sum(1 for s in st2 if s["status"] & 3),
                    "eager_ms_per_step_same_state": eager_same_state}
    pairs = float(sum(s["n_targets"] * s["num_samples"] for s in st2))
    out["batch"]["far_pairs_per_step"] = pairs
    sizes = [s["n_fluid"] for s in st2]
    out["scene_fluid_min_median_max"] = [int(np.min(sizes)), int(np.median(sizes)), int(np.max(sizes))]
    del b
    torch.cuda.synchronize()
    # one scene at a time
    from .particle_system import ParticleSystem
    solvers = []
    for cfg in cfgs:
        ps = ParticleSystem(cfg)
        sv = ps.build_solver()
        sv.initialize()
        solvers.append((ps, sv))
    for ps, sv in solvers:
        for _ in range(2):
            sv.step()
    torch.cuda.synchronize()
    lat = np.zeros((lone_rounds, len(solvers)))
    nfl = np.zeros(len(solvers))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_all = 0.0
    for r in range(lone_rounds):
        for k, (ps, sv) in enumerate(solvers):
            e0.record()
            sv.step()
            e1.record()
            e1.synchronize()
            lat[r, k] = e0.elapsed_time(e1)
    for k, (ps, sv) in enumerate(solvers):
        nfl[k] = ps.fluid_particle_num[None]
    t_round = lat.sum(1).mean()
    out["one_at_a_time"] = {"ms_per_round": float(t_round),
                            "particle_steps_per_s": float(nfl.sum() / (t_round * 1e-3)),
                            "latency_ms_p50": float(np.percentile(lat, 50)),
                            "latency_ms_p99": float(np.percentile(lat, 99))}
    out["batch_speedup"] = out["batch"]["particle_steps_per_s"] / out["one_at_a_time"]["particle_steps_per_s"]
    return out


def single_scene_latency(steps: int = 50, warmup: int = 5) -> dict:
    """The small channel (10k fluid, r = 0.01) stepped alone: the host-driven
    KarmanVortexSolver.step() against the same scene as a batch of one whose
    steps replay from a CUDA graph (device emission, device Jacobi loops)."""
    from . import scenes
    from .particle_system import ParticleSystem
    cfg = scenes.channel2d(trim_cylinder=True)
    cfg.config["Configuration"]["computeVis"] = False
    ps = ParticleSystem(cfg)
    sv = ps.build_solver()
    sv.initialize()
    for _ in range(warmup):
        sv.step()
    lone = _ev_time(sv.step, steps)
    n_fluid = ps.fluid_particle_num[None]
    del sv, ps
    b = SceneBatch([cfg])
    for _ in range(warmup):
        b.step()
    eager = _ev_time(b.step, 10)
    b.capture(2)
    b.replay()
    graph = _ev_time(b.replay, steps // 2) / 2
    return {"workload": "small channel, 1 scene", "fluid_particles": int(n_fluid),
            "lone_step_ms": lone, "batch_of_one_eager_ms": eager, "batch_of_one_graph_ms": graph,
            "graph_speedup_vs_lone": lone / graph}


def profile_window(n_scenes: int = 256, seed: int = 0, warmup: int = 6, steps: int = 2, tile: int = 2):
    """Eager batch steps bracketed by cudaProfilerStart/Stop, for a profiler
    started with --profile-from-start off."""
    cfgs, _ = channel_batch_configs(n_scenes=n_scenes, seed=seed)
    b = SceneBatch(cfgs)
    b._check(b.lib.dv_set_far_tile(b.ctx, int(tile)), "dv_set_far_tile")
    for _ in range(warmup):
        b.step()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    for _ in range(steps):
        b.step()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    return b.states()


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--scenes", type=int, default=256)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--out", type=str, default=None)
    ap.add_argument("--single", action="store_true", help="only the one-scene latency comparison")
    ap.add_argument("--profile-window", action="store_true",
                    help="only run 2 eager steps inside cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    a = ap.parse_args()
    if a.single:
        print(json.dumps(single_scene_latency()))
        return
    if a.profile_window:
        st = profile_window(n_scenes=a.scenes)
        print(json.dumps({"profiled_steps": 2, "scenes": len(st)}))
        return
    res = run(n_scenes=a.scenes, reps=a.reps)
    s = json.dumps(res)
    print(s)
    if a.out:
        with open(a.out, "w") as f:
            f.write(s + "\n")


if __name__ == "__main__":
    main()
