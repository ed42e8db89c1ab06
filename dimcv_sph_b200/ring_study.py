"""Operator-level MC-VVPE versus full Biot-Savart on the 3-D vortex ring.

N particles uniform in [-1,1]³ carry a Gaussian-core ring vorticity plus
noise; the velocity that feeds KVN comes from one FP32 full Biot-Savart pass.
One MC-VVPE step is: grid rebuild, the fused ∇v sweep (KVN), AKDE, FP64-CDF
inverse-CDF sampling of M particles, and the VVPE (near-field neighbour sum +
Monte-Carlo far field).  One full-BS step is: grid rebuild and the O(N²)
FP32 sum.  Errors are RMS over a fixed subset of targets against the FP64
full Biot-Savart sum (computed on the GPU in double precision).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib, scenes
from ._abi import DV_SAMPLE_INVERSE_CDF, DV_SAMPLE_STRATIFIED
from .dimcv_sph import DIMCVSPHSolver
from .particle_system import ParticleSystem


class RingStudy:
    def __init__(self, n: int = 1 << 20, seed: int = 0, subset: int = 262144, device="cuda",
                 kernel3d: bool = True):
        cfg, x, w = scenes.ring3d(n, seed, kernel3d=kernel3d)
        ps = ParticleSystem(cfg, device=device, capacity=n)
        z = np.zeros_like(x)
        ps.add_particles(0, n, x, z, np.full(n, 1000.0), np.zeros(n), np.ones(n, np.int32),
                         np.ones(n, np.int32), np.zeros((n, 3), np.int32))
        solver = DIMCVSPHSolver(ps)
        solver.initialize()
        self.ps, self.solver, self.n = ps, solver, n
        perm = ps.permutation()
        dev = ps.device
        self.omega = torch.zeros((ps.particle_max_num, 4), dtype=torch.float32, device=dev)
        self.omega[:n, :3] = torch.from_numpy(w[perm]).to(dev)
        solver.d_vort_smoothed[:n] = self.omega[:n, :3]
        u = self.bs(None, n, 32)
        ps.v[:n] = u[:, :3]
        self.v0 = ps.v[:n].clone()
        rng = np.random.default_rng(seed + 1)
        sub = np.sort(rng.choice(n, size=min(subset, n), replace=False)).astype(np.int32)
        self.sub = torch.from_numpy(sub).to(dev)
        self.uref = self.bs(self.sub, len(sub), 64)[:, :3]
        self.uref_rms = float(torch.sqrt((self.uref ** 2).sum(1).mean()))

    def bs(self, targets, nt, precision):
        ps = self.ps
        out = torch.zeros((nt, 4), dtype=torch.float64 if precision == 64 else torch.float32, device=ps.device)
        tp = C.c_void_p(targets.data_ptr()) if targets is not None else None
        rc = ps.lib.dv_bs_full(ps.ctx, C.byref(ps.fields_struct), C.c_void_p(self.omega.data_ptr()), tp, nt,
                               C.c_void_p(out.data_ptr()), precision)
        _lib.check(ps.ctx, rc, "dv_bs_full")
        return out

    def set_compensated(self, on: bool):
        ps = self.ps
        ps.params.compensated = 1 if on else 0
        _lib.check(ps.ctx, ps.lib.dv_set_params(ps.ctx, C.byref(ps.params)), "dv_set_params")

    def mc_step(self, M: int, seed_step: int, mode: int = DV_SAMPLE_INVERSE_CDF, restore: bool = True):
        """One MC-VVPE step from the ring's initial velocity (restore) or from
        the velocity the last step left; the work of a step (pairs, sweeps)
        does not depend on which, so the timings skip the restore."""
        ps, s = self.ps, self.solver
        if restore:
            ps.v[: self.n] = self.v0
        ps.initialize_particle_system()
        s._calls("dv_dimcv_vorticity")  # ∇v for KVN (the step's Δω is not used here)
        s.compute_kinematic_vorticity_num_sample()
        s.compute_kernel_density()
        s._calls("dv_sample", mode, s.seed, seed_step, int(M))
        s.vort2vel()

    def bs_step(self):
        self.ps.initialize_particle_system()
        return self.bs(None, self.n, 32)

    def mc_error(self) -> float:
        got = self.solver.v_vort[self.sub.long()].double()
        return float(torch.sqrt(((got - self.uref) ** 2).sum(1).mean())) / self.uref_rms

    def timed(self, fn, reps: int) -> float:
        """ms per call on the device (CUDA events on the current stream)."""
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps


def run(n=1 << 20, Ms=(4096, 16384, 32768, 40960, 49152, 51200, 53248, 57344, 65536, 131072), seeds=8,
        subset=262144, reps=3, target_err=0.02, tune_M=49152, device="cuda") -> dict:
    st = RingStudy(n=n, subset=subset, device=device)
    out = {"n": n, "subset": int(st.sub.numel()), "kernel": "blob3d (1/4π) V (r×ω)/(|r|²+δ²)^{3/2}, δ = r",
           "bs_f32_vs_f64": {}, "mc": []}
    # FP32 accumulation error of the full sum, plain and compensated
    for comp in (False, True):
        st.set_compensated(comp)
        u32 = st.bs(st.sub, st.sub.numel(), 32)[:, :3].double()
        err = float(torch.sqrt(((u32 - st.uref) ** 2).sum(1).mean())) / st.uref_rms
        out["bs_f32_vs_f64"]["compensated" if comp else "plain"] = err
    st.set_compensated(False)
    # the full-BS step at its best far tile (the paired loop's 4, 6 or 8
    # targets per thread); the MC steps below autotune their own
    lib, ctx = st.ps.lib, st.ps.ctx
    tiles = {}
    for tt in (4, 6, 8):
        _lib.check(ctx, lib.dv_set_far_tile(ctx, tt), "dv_set_far_tile")
        tiles[tt] = st.timed(st.bs_step, 1)
    best = min(tiles, key=tiles.get)
    _lib.check(ctx, lib.dv_set_far_tile(ctx, best), "dv_set_far_tile")
    bs_ms = st.timed(st.bs_step, 2)
    out["bs_step_ms"] = bs_ms
    out["bs_far_tile"] = best
    out["bs_tile_sweep_ms"] = {str(k): v for k, v in tiles.items()}
    out["bs_particle_steps_per_s"] = n / (bs_ms * 1e-3)
    out["bs_tflops_incl_grid"] = 27.0 * n * (n - 1) / (bs_ms * 1e-3) / 1e12
    # the MC steps' far tile: the autotuner's choice at tune_M samples, near
    # the matched error, instead of at the first M of the sweep
    st.solver.far_tile = None
    st.mc_step(tune_M, 999, DV_SAMPLE_STRATIFIED)
    out["mc_far_tile"] = st.solver.far_tile
    out["mc_far_tile_tuned_at_M"] = tune_M
    for mode_name, mode in (("iid", DV_SAMPLE_INVERSE_CDF), ("stratified", DV_SAMPLE_STRATIFIED)):
        for M in Ms:
            errs = []
            for k in range(seeds):
                st.mc_step(M, 1000 + k, mode)
                errs.append(st.mc_error())
            st.mc_step(M, 7, mode)
            ms = st.timed(lambda: st.mc_step(M, 7, mode, restore=False), reps)
            st.set_compensated(True)
            st.mc_step(M, 1000, mode)
            err_comp = st.mc_error()
            st.set_compensated(False)
            out["mc"].append({"sampler": mode_name, "M": M, "rms_err_mean": float(np.mean(errs)),
                              "rms_err_std": float(np.std(errs)), "rms_err_compensated_seed0": err_comp,
                              "step_ms": ms, "particle_steps_per_s": n / (ms * 1e-3),
                              "speedup_vs_bs": bs_ms / ms})
    out["target_rms_err"] = target_err
    out["matched"] = {}
    for mode_name in ("iid", "stratified"):
        ok = [m for m in out["mc"] if m["sampler"] == mode_name and m["rms_err_mean"] <= target_err]
        out["matched"][mode_name] = min(ok, key=lambda m: m["M"]) if ok else None
    return out


def main():
    import argparse
    import json
    ap = argparse.ArgumentParser(description="MC-VVPE vs full Biot-Savart on the 3-D vortex ring")
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--seeds", type=int, default=8)
    ap.add_argument("--bs-only", action="store_true",
                    help="only build the ring and run the FP32 full Biot-Savart sum --reps times (a small case "
                         "for a profiler capture of the paired blob loop)")
    ap.add_argument("--tile", type=int, default=6, help="targets per thread of the paired loop (--bs-only)")
    ap.add_argument("--reps", type=int, default=2)
    a = ap.parse_args()
    if a.bs_only:
        st = RingStudy(n=a.n, subset=min(1024, a.n))
        _lib.check(st.ps.ctx, st.ps.lib.dv_set_far_tile(st.ps.ctx, a.tile), "dv_set_far_tile")
        for _ in range(a.reps):
            st.bs(None, st.n, 32)
        torch.cuda.synchronize()
        print(json.dumps({"n": a.n, "tile": a.tile, "bs_ms": st.timed(lambda: st.bs(None, st.n, 32), a.reps)}))
        return
    print(json.dumps(run(n=a.n, seeds=a.seeds)))


if __name__ == "__main__":
    main()
