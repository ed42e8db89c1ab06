#!/usr/bin/env python
"""DIMCV-SPH step throughput on B200: particle-steps/s of the full
DFSPH + MC-VVPE step (grid rebuild, density/divergence solves, KVN/AKDE
sampling, Monte-Carlo Biot-Savart VVPE) on the 3-D sphere scene
(~2.0M fluid + ~0.3M boundary particles, M = N/32 samples).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sphere3d|channel2d]

One process per GPU (torchrun for N > 1).  The path does not exchange data
between GPUs, so N > 1 runs independent replicas ("replicas only"); the
only collectives are a barrier and a MAX of the device-timed elapsed time.
Inputs are synthetic (seeded lattice scenes); the state (~1.3 GB) is larger
than L2, so no explicit L2 flush is done between steps.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/s (DFSPH+MC-VVPE) vs full Biot-Savart on 1 B200 at equal vel. error"
UNIT = "particle-steps/s"
# algorithmic FP32 operations per (target, sample) pair of the far field:
# the reference kernel in 2-D and 3-D, and the 3-D blob kernel (+3)
FLOPS_PER_PAIR = {2: 12, 3: 24}
FLOPS_PER_PAIR_BLOB = 27


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)  # the sphere configuration's 100 steps
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["sphere3d", "channel2d"], default="sphere3d")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-vs-bs", action="store_true",
                    help="skip the MC-VVPE vs full Biot-Savart study on the 1M-particle vortex ring")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU time of the baseline sample")
    ap.add_argument("--scale", type=float, default=1.0, help="particle radius multiplier (1 = benchmark size)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the extra figures: the sphere with the 3-D blob kernel, the 256-scene batch "
                         "and the adjoint rollout")
    ap.add_argument("--far-tile", type=int, default=None,
                    help="far-field targets per thread (2, 4, 6, 8) instead of the autotuner's choice")
    ap.add_argument("--far-chunks", type=int, default=None, help="far-field sample chunks (1..8)")
    return ap.parse_args()


def workload_config(name, scale=1.0):
    """scale multiplies the particle radius (and dt): 1 is the benchmark
    configuration; 2 is the 8x smaller case used for detailed ncu captures."""
    from dimcv_sph_b200 import scenes
    if name == "sphere3d":
        r = 0.004 * scale
        return scenes.sphere3d(radius=r, dt=1.6e-4 * scale), {
            "workload": f"sphere3d: flow past a sphere r=0.15 in a 3x1x1 box, r={r:g} (h={4 * r:g}), "
                        f"inflow 1 m/s, M=N/32 inverse-CDF samples, dt={1.6e-4 * scale:g}, FP32 state, seed 0"}
    r = 0.01 * scale
    return scenes.channel2d(radius=r, dt=4e-4 * scale), {
        "workload": f"channel2d: 2-D von Karman channel [0,4]x[0,1], r={r:g}, cylinder r=0.1, inflow 1 m/s, "
                    f"M=N/16, dt={4e-4 * scale:g}, seed 0"}


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.proc = None
        self.ident = str(device_index)
        try:
            import torch
            uuid = getattr(torch.cuda.get_device_properties(device_index), "uuid", None)
            if uuid is not None:
                self.ident = "GPU-" + str(uuid)
        except Exception:
            pass

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", self.ident], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [t.strip() for t in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


# ----------------------------------------------------------- distributed
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def _all_reduce(x: float, world: int, op: str) -> float:
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float, world: int) -> float:
    return _all_reduce(x, world, "max")


def aggregate_throughput(ms_local: float, units_local: float, world: int):
    """Whole-job throughput of weakly scaled replicas: the units every rank
    processed, over the slowest rank's device time.  Returns (ms, units/s)."""
    ms = _all_reduce(ms_local, world, "max")
    units = _all_reduce(units_local, world, "sum")
    return ms, units / (ms * 1e-3)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------------- our arm
STAGES = {
    "grid": ["initialize_particle_system"],
    "dfsph": ["compute_densities", "compute_DFSPH_factor", "divergence_solve", "compute_non_pressure_forces",
              "predict_velocity", "pressure_solve"],
    "dimcv_sweeps": ["init", "compute_d_vorticity", "compute_all_d_vort_smoothed", "update_sample",
                     "compute_kernel_density", "smooth_and_kernel_density", "_draw_samples"],
    "vvpe": ["vort2vel"],
    "integrate_vis": ["update_particle_life_time", "copy_x_temp", "advect"],
}


# Algorithmic HBM bytes per particle slot of each stage (3-D; 2-D uses d = 2
# in the vector terms): per sweep of the reference, every field it needs read
# once and every field it produces written once, neighbour re-reads excluded
# (a fused walk reads the fields its sweeps share once, so it moves fewer).  Grid: x, keys and
# the permuted persistent set (96); DFSPH: densities 21, factor 25, density
# change 33 (+ 57 + 33 per divergence iteration), non-pressure 41, predict 36,
# density_adv 33 (+ 57 + 33 per pressure iteration); DIMCV: fused grad-v /
# curl / KVN / delta-omega 57, smoothing 40, AKDE 20, CDF 12.  The far field is
# FP32-bound and has its own roofline.
def stage_bytes(dim: int, it_div: int, it_p: int) -> dict:
    s = 1.0 if dim == 3 else 2.0 / 3.0  # vector fields shrink with d
    return {"grid": 96 * s,
            "dfsph": (21 + 25 + 33 + 90 * it_div + 41 + 36 + 33 + 90 * it_p) * s,
            "dimcv_sweeps": (57 + 40 + 20 + 12) * s}


def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (copy bandwidth)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def stage_roofline(st: dict, dim: int, slots: int, it_div: int, it_p: int) -> dict:
    peak, src = hbm_peak()
    out = {"peak_gbs": peak, "peak_source": src, "unit": "GB/s", "stages": {}}
    for k, b in stage_bytes(dim, it_div, it_p).items():
        ms = st.get(k, 0.0)
        if ms > 0:
            gbs = b * slots / (ms * 1e-3) / 1e9
            out["stages"][k] = {"alg_bytes_per_slot": round(b, 1), "achieved": round(gbs, 1),
                                "frac": round(gbs / peak, 4)}
    return out


def stage_times(solver, ps, steps: int) -> dict:
    """Per-stage device time of `steps` steps (CUDA events on the solver's
    stream around each reference method; outside the timed region)."""
    import torch
    acc = {k: 0.0 for k in STAGES}
    wrapped = []
    evs = []

    def wrap(obj, name, stage):
        orig = getattr(obj, name)

        def w(*a, **k):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r = orig(*a, **k)
            e1.record()
            evs.append((stage, e0, e1))
            return r
        setattr(obj, name, w)
        wrapped.append((obj, name))

    for stage, names in STAGES.items():
        for nm in names:
            wrap(ps if nm == "initialize_particle_system" else solver, nm, stage)
    try:
        for _ in range(steps):
            solver.step()
        torch.cuda.synchronize()
        for stage, e0, e1 in evs:
            acc[stage] += e0.elapsed_time(e1)
    finally:
        for obj, name in wrapped:
            delattr(obj, name)
    return {k: v / steps for k, v in acc.items()}


def far_traffic(workload: str, tile: int, chunks: int, n_targets: float):
    """DRAM bytes (read + write) per far-field launch: from the committed
    capture record of the same workload, tile and sample-chunk count
    (profiles/far_field_traffic.json, an ncu capture of the 8x smaller case),
    scaled by the targets of one launch; None when no record matches."""
    p = ROOT / "profiles" / "far_field_traffic.json"
    try:
        recs = json.loads(p.read_text())["captures"]
    except (OSError, KeyError, ValueError):
        return None
    for r in recs:
        if r["workload"] == workload and r["far_tile"] == tile and r["far_chunks"] == chunks:
            return {"bytes_per_launch": r["dram_bytes_per_launch"] * n_targets / r["n_targets"],
                    "capture": {k: r[k] for k in ("scale", "n_targets", "num_samples", "dram_bytes_per_launch",
                                                  "command")},
                    "scaled_by": "targets per launch (target reads and partial writes grow with them; the "
                                 "samples stay L2-resident)"}
    return None


def vvpe_applied(ps, solver) -> dict:
    """One step with the VVPE's effect counted: the fluid rows whose velocity
    the gate |v_vort| < |v| (dimcv_sph.py:717-719) let the VVPE change, and
    the rows with a finite v_vort."""
    import torch
    orig = solver.vort2vel
    rec = {}

    def tap():
        n = ps.particle_num[None]
        before = ps.v[:n].clone()
        orig()
        fl = ps.material[:n] == 1
        changed = ((ps.v[:n] != before).any(1) & fl).sum()
        finite = (torch.isfinite(solver.v_vort[:n]).all(1) & fl).sum()
        rec.update(fluid=int(fl.sum()), applied=int(changed), finite=int(finite))

    solver.vort2vel = tap
    try:
        solver.step()
    finally:
        del solver.vort2vel
    return {"fraction": rec["applied"] / max(1, rec["fluid"]), "finite_fraction": rec["finite"] / max(1, rec["fluid"]),
            "fluid_rows": rec["fluid"]}


def set_far_shape(args, ps, solver):
    from dimcv_sph_b200 import _lib
    if args.far_tile:
        solver.far_tile = args.far_tile
        _lib.check(ps.ctx, ps.lib.dv_set_far_tile(ps.ctx, args.far_tile), "dv_set_far_tile")
    if args.far_chunks:
        _lib.check(ps.ctx, ps.lib.dv_set_far_chunks(ps.ctx, args.far_chunks), "dv_set_far_chunks")


def kernel3d_figure(args, steps: int = 10) -> dict:
    """The sphere workload with the regularised 3-D blob kernel in place of
    the reference's 2-D projected one (no 0/0 rows, so every fluid row's far
    field reaches v through the gate test): particle-steps/s and the far
    field's FP32 roofline."""
    import torch
    from dimcv_sph_b200.particle_system import ParticleSystem
    cfg, config = workload_config(args.workload, args.scale)
    cfg.config["Configuration"]["kernel3D"] = True
    ps = ParticleSystem(cfg)
    solver = ps.build_solver()
    solver.initialize()
    set_far_shape(args, ps, solver)
    lib, ctx = ps.lib, ps.ctx
    peak = C.c_double(0)
    lib.dv_fp32_peak(ctx, C.byref(peak))
    for _ in range(3):
        solver.step()
    torch.cuda.synchronize()
    cnt0 = ps.counters()
    lib.dv_profile(ctx, 1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        solver.step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    far_ms, far_launches, pairs = C.c_double(), C.c_int64(), C.c_double()
    lib.dv_profile_read(ctx, C.byref(far_ms), C.byref(far_launches), C.byref(pairs))
    lib.dv_profile(ctx, 0)
    cnt1 = ps.counters()
    n_fluid = 0.5 * (cnt0["n_fluid"] + cnt1["n_fluid"])
    ach = FLOPS_PER_PAIR_BLOB * pairs.value / (far_ms.value * 1e-3) / 1e12 if far_ms.value > 0 else 0.0
    out = {"workload": config["workload"] + "; kernel3D: blob (1/4π) V (ω×r)/(|r|²+δ²)^{3/2}, δ = r",
           "value": n_fluid * steps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
           "far_field": {"achieved": round(ach, 3), "peak": round(peak.value / 1e12, 3), "unit": "TFLOP/s",
                         "frac": round(ach / (peak.value / 1e12), 4) if peak.value else None,
                         "flops_per_pair": FLOPS_PER_PAIR_BLOB, "kernel_ms_per_step": far_ms.value / steps,
                         "far_tile_targets_per_thread": solver.far_tile,
                         "far_sample_chunks": int(lib.dv_get_far_chunks(ctx))},
           "vvpe_applied": vvpe_applied(ps, solver)}
    return out


def run_ours(args, rank, world, local):
    import torch
    from dimcv_sph_b200 import _lib
    from dimcv_sph_b200.particle_system import ParticleSystem

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    cfg, config = workload_config(args.workload, args.scale)
    ps = ParticleSystem(cfg, device=dev)
    solver = ps.build_solver()
    solver.initialize()
    set_far_shape(args, ps, solver)
    lib, ctx = ps.lib, ps.ctx
    peak = C.c_double(0)
    _lib.check(ctx, lib.dv_fp32_peak(ctx, C.byref(peak)), "dv_fp32_peak")
    for _ in range(max(3, args.warmup)):
        solver.step()
    torch.cuda.synchronize()
    cnt0 = ps.counters()
    lib.dv_profile(ctx, 1)
    launches0 = lib.dv_launch_count(ctx)
    clocks = ClockSampler(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        solver.step()
    e1.record()
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms_local = e0.elapsed_time(e1)
    launches = lib.dv_launch_count(ctx) - launches0
    far_ms, far_launches, pairs = C.c_double(), C.c_int64(), C.c_double()
    lib.dv_profile_read(ctx, C.byref(far_ms), C.byref(far_launches), C.byref(pairs))
    lib.dv_profile(ctx, 0)
    cnt1 = ps.counters()
    n_fluid = 0.5 * (cnt0["n_fluid"] + cnt1["n_fluid"])
    ms, value = aggregate_throughput(ms_local, n_fluid * args.steps, world)

    # dominant kernel roofline (Monte-Carlo far field, FP32-pipe bound)
    dim = ps.dim
    achieved = FLOPS_PER_PAIR[dim] * pairs.value / (far_ms.value * 1e-3) / 1e12 if far_ms.value > 0 else 0.0
    peak_tf = peak.value / 1e12
    far_chunks = int(ps.lib.dv_get_far_chunks(ps.ctx))
    tr = far_traffic(args.workload if args.scale == 1.0 else f"{args.workload}@{args.scale:g}", solver.far_tile,
                     far_chunks, cnt1["n_targets"])
    roofline = {"kernel": "k_far_main (Monte-Carlo Biot-Savart far field)", "bound": "fp32",
                "achieved": round(achieved, 3), "peak": round(peak_tf, 3), "unit": "TFLOP/s",
                "frac": round(achieved / peak_tf, 4) if peak_tf else None,
                "traffic": tr["bytes_per_launch"] if tr else None,
                "peak_source": "measured in this run: FP32 FMA chain kernel (dv_fp32_peak), an FMA counts 2",
                "flops_per_pair": FLOPS_PER_PAIR[dim], "pairs_per_step": pairs.value / args.steps,
                "kernel_ms_per_step": far_ms.value / args.steps,
                "kernel_share_of_step": far_ms.value / ms_local}
    if tr:
        roofline["traffic_source"] = tr

    result = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
              "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True,
              "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
              "config": dict(config, n_particles=cnt1["n"], n_fluid=cnt1["n_fluid"],
                             num_samples=cnt1["num_samples"], parallelism=f"replicas x{world}",
                             l2="state (~1.3 GB) larger than L2; no flush"),
              "clocks": clk, "gpu_launches": int(launches), "roofline": roofline,
              "iterations": {"divergence": cnt1["iters_div"], "pressure": cnt1["iters_p"]},
              "far_tile_targets_per_thread": solver.far_tile,
              "far_sample_chunks": far_chunks}

    # per-stage device times and HBM fractions (outside the timed region)
    st = stage_times(solver, ps, 3)
    result["stages_ms"] = {k: round(v, 3) for k, v in st.items()}
    cnt2 = ps.counters()
    result["stage_roofline"] = stage_roofline(st, dim, cnt2["n"], cnt2["iters_div"], cnt2["iters_p"])

    # the share of fluid rows whose velocity the VVPE changes (one more step)
    result["vvpe_applied_fraction"] = vvpe_applied(ps, solver)
    if not args.no_e2e:
        result["e2e"] = e2e(args, ps, solver, world)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(args, ps, solver)
    if rank == 0 and world == 1:
        del ps, solver
        torch.cuda.empty_cache()
        if not args.no_extras and args.workload == "sphere3d":
            result["kernel3d"] = kernel3d_figure(args)
            torch.cuda.empty_cache()
        if not args.no_vs_bs:
            from dimcv_sph_b200 import ring_study
            result["vs_full_bs"] = ring_study.run(n=1 << 20)
            torch.cuda.empty_cache()
        if not args.no_extras:
            from dimcv_sph_b200 import adjoint_study, batch_study
            result["batch_c4"] = batch_study.run(lone_rounds=2)
            torch.cuda.empty_cache()
            result["adjoint_c3"] = adjoint_study.timing()
            torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def e2e(args, ps, solver, world):
    """The same metric through the public API (KarmanVortexSolver.step) with
    the state round-tripped through pinned host buffers every step: H2D of
    x and v before the step, D2H of x and v after it, inside the timed region.
    The host buffers have the reference's field shape, (capacity, dim) float32
    (particle_system.py:153-154), and are copied through the ps.x / ps.v views
    of the device's padded rows."""
    import torch
    cap = ps.particle_max_num
    vs = ps.x.shape[1]
    hx = torch.empty((cap, vs), dtype=torch.float32, pin_memory=True)
    hv = torch.empty((cap, vs), dtype=torch.float32, pin_memory=True)
    hx.copy_(ps.x)
    hv.copy_(ps.v)
    torch.cuda.synchronize()
    steps = args.steps
    cnt0 = ps.counters()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        ps.x.copy_(hx, non_blocking=True)
        ps.v.copy_(hv, non_blocking=True)
        solver.step()
        hx.copy_(ps.x, non_blocking=True)
        hv.copy_(ps.v, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    cnt1 = ps.counters()
    n_fluid = 0.5 * (cnt0["n_fluid"] + cnt1["n_fluid"])
    nbytes = 2 * cap * vs * 4
    return {"value": world * n_fluid * steps / (ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": nbytes,
            "api": "KarmanVortexSolver.step() with x, v (capacity x dim float32 each, the reference's field "
                   "shape) copied from/to pinned host memory each step"}


# ----------------------------------------------------------- CPU baseline
def oracle_from_gpu(ps, solver):
    from oracle.oracle import OracleSim
    o = OracleSim(ps.params, ps.particle_max_num, 0)
    o.load_snapshot(ps.snapshot(), ps.counters())
    return o


def timed_sample(o, lo, hi, it_div, it_p, M, compute_vis=True):
    """One substep restricted to slots [lo, hi) on the oracle; seconds."""
    o.lib.dvo_set_sample(o.ctx, lo, hi, it_div, it_p)
    t0 = time.perf_counter()
    o.substep(sampler="injected", M=M, compute_vis=compute_vis, vvpe_precision=32)
    return time.perf_counter() - t0


def sample_fluid(o, lo, hi):
    return int(np.count_nonzero(o.f["material"][lo:hi] == 1))


def cpu_baseline(args, ps, solver):
    """The CPU oracle (a C++/OpenMP restatement of the reference kernels,
    "port") on the host cores: the grid rebuild of the full state is timed
    once and charged pro rata; one substep runs on a contiguous slot range
    (a spatially compact Morton block) with the GPU's iteration counts and its
    M samples, sized to about --cpu-seconds of CPU work."""
    ps.initialize_particle_system()
    cnt = ps.counters()
    o = oracle_from_gpu(ps, solver)
    n = cnt["n"]
    t0 = time.perf_counter()
    o.counting_sort()
    t_sort = time.perf_counter() - t0
    M = cnt["num_samples"]
    it_div, it_p = max(1, cnt["iters_div"]), max(1, cnt["iters_p"])
    # a short probe sizes the sample; the sample runs on the next, disjoint range
    probe = min(n // 4, 2048)
    t_probe = timed_sample(o, n // 4, n // 4 + probe, it_div, it_p, M)
    per = t_probe / max(1, probe)
    lo = n // 4 + probe
    S = int(min(n - lo, max(probe, args.cpu_seconds / max(per, 1e-9))))
    t = timed_sample(o, lo, lo + S, it_div, it_p, M)
    nf = sample_fluid(o, lo, lo + S)
    t_total = t + t_sort * S / n
    return {"value": nf / t_total, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"1 substep on {S} of {n} slots (contiguous Morton range, {nf} fluid) with the GPU's "
                      f"{M} samples and iteration counts ({it_div}, {it_p}); full grid rebuild {t_sort:.2f}s "
                      f"charged pro rata; {t_total:.1f}s CPU wall"}


# ------------------------------------------------------- reference arm
def oracle_scene(cfg):
    """The workload built on the host only (no GPU): lattices as the
    ParticleSystem builds them, loaded into the CPU oracle."""
    from dimcv_sph_b200.params import Options, make_params
    from oracle.oracle import OracleSim
    from dimcv_sph_b200.particle_system import ParticleSystem
    g = cfg.get_cfg
    dim = len(g("domainStart"))
    r = g("particleRadius")
    m_V0 = float(np.float32(0.8 * (2 * r) ** dim))
    helper = ParticleSystem.__new__(ParticleSystem)
    helper.dim = dim
    helper.particle_diameter = 2 * r
    blocks = [(b, 1) for b in cfg.get_fluid_blocks()] + [(b, 0) for b in cfg.get_rigid_blocks()]
    arrays = []
    for b, mat in blocks:
        off = np.array(b.get("translation", [0.0] * dim))
        start = np.array(b["start"]) + off
        end = np.array(b["end"]) + off
        pos = helper._lattice(start, (end - start) * np.array(b.get("scale", [1] * dim)), helper._exclusion(b))
        vel = np.tile(np.asarray(b["velocity"], np.float32)[:dim], (pos.shape[0], 1))
        arrays.append((b, mat, pos, vel))
    cap = sum(a[2].shape[0] for a in arrays) + int(g("reservedCapacity") or 0)
    o = OracleSim(make_params(cfg, Options.from_config(cfg)), cap, 0)
    for b, mat, pos, vel in arrays:
        o.add_particles(pos, vel, b["objectId"], float(np.float32(b["density"])), 0.0, mat, int(mat == 1),
                        tuple(b["color"]), m_V0)
    o.initialize_particle_system()
    o.call("boundary_volume")
    return o


def jacobi_counts(o):
    """Iteration counts of the divergence and pressure solves on the full
    state (densities, factor, divergence solve, non-pressure forces,
    prediction, pressure solve; the VVPE's small velocity change before the
    pressure solve is left out).  Returns (it_div, it_p, seconds)."""
    t0 = time.perf_counter()
    o.lib.dvo_set_sample(o.ctx, 0, 0x7FFFFFFF, 0, 0)
    snap = {k: o.f.a[k].copy() for k in ("v", "density", "dfsph_factor", "density_adv", "acceleration")}
    o.call("densities")
    o.call("dfsph_factor")
    it_div = o.divergence_solve()
    o.call("nonpressure")
    o.call("predict_velocity")
    it_p = o.pressure_solve()
    for k, a in snap.items():
        o.f.a[k][...] = a
    return max(1, it_div), max(1, it_p), time.perf_counter() - t0


def run_reference(args, rank, world):
    """The reference's CPU path on the host cores.  Taichi (the reference's
    runtime) is not installable here, so the arm runs the oracle port: each
    step is one substep on a bounded slot range of the same workload (all
    threads), its fluid particle count / time being the line's value."""
    if rank != 0:
        return
    cfg, config = workload_config(args.workload, args.scale)
    o = oracle_scene(cfg)
    n = o.counters()["n"]
    t0 = time.perf_counter()
    o.counting_sort()
    t_sort = time.perf_counter() - t0
    n_fluid = o.counters()["n_fluid"]
    M = max(1, int(n_fluid / 32)) if args.workload == "sphere3d" else max(1, int(n_fluid / 16))
    # samples: M uniform fluid slots (the draw itself is O(M log N), negligible)
    rng = np.random.default_rng(0)
    fl = np.nonzero(o.f["material"][:n] == 1)[0]
    smp = np.sort(rng.choice(fl, size=M, replace=False)).astype(np.int32)
    o.solver["sample_idx"][:M] = smp
    it_div, it_p, t_solve = jacobi_counts(o)
    budget = max(1.0, 120.0 / max(1, args.steps + args.warmup))
    lo = n // 3
    probe = min(n - lo, 1024)
    per = timed_sample(o, lo, lo + probe, it_div, it_p, M) / probe
    S = int(min(n - lo, max(probe, budget / max(per, 1e-9))))
    tot_t, tot_p = 0.0, 0
    for k in range(args.warmup + args.steps):
        a = lo + (k * S) % max(1, n - lo - S + 1)
        t = timed_sample(o, a, a + S, it_div, it_p, M) + t_sort * S / n
        if k >= args.warmup:
            tot_t += t
            tot_p += sample_fluid(o, a, a + S)
    value = tot_p / tot_t
    sample = (f"each step: 1 substep on {S} of {n} slots (contiguous Morton range) with {M} samples and "
              f"{it_div}+{it_p} Jacobi iterations (measured by one full-state solve, {t_solve:.1f}s); "
              f"full grid rebuild {t_sort:.2f}s charged pro rata")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / max(1, args.steps), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": config,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "Taichi (the reference runtime) is not installed and cannot be; the reference arm is the "
                    "C++/OpenMP restatement of the reference kernels in oracle/"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
