"""Inverse-problem study on the periodic 2-D box (differentiable rollout).

Workload: [0,1]² periodic, n particles on a jittered √n × √n lattice
(jitter U(-0.25, 0.25)·spacing), initial vorticity 8 Gaussian blobs
(amplitude N(0, 5), σ ~ U(0.03, 0.08)); a 32-step rollout (dt 0.01) with
checkpoints every 8 steps; loss = mean |u_32 − u*|² against the final
velocity of a full Biot-Savart rollout from blobs of another seed.

Reports (one JSON object):
  * forward and adjoint (backward incl. recompute) device times and ratio,
    per-step plan / operator / VJP times;
  * FP64 adjoint vs FP64 central differences (ε = 1e-6) on 64 coordinates,
    plans and periodic images frozen;
  * FP32 adjoint vs FP64 adjoint on the same frozen plans;
  * MC adjoint vs the full Biot-Savart adjoint: one gradient and the mean of
    R independent sampler streams (unbiasedness: error ~ R^-1/2), and one
    stream with M from N/16 to N samples per step (error and cost);
  * Adam on the initial vorticity with MC gradients and with full-BS
    gradients, the loss measured with the full Biot-Savart forward.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import scenes
from .adjoint import FULL, MC, VortexBox, fd_check, timed


def _nrel(a, b):
    a = torch.as_tensor(a).double()
    b = torch.as_tensor(b).double()
    return float((a - b).norm() / b.norm())


def _cos(a, b):
    a = torch.as_tensor(a).double()
    b = torch.as_tensor(b).double()
    return float((a * b).sum() / (a.norm() * b.norm()))


def timing(n: int = 65536, steps: int = 32, ckpt: int = 8, mc_fraction: float = 1.0 / 16.0, seed: int = 0,
           target_seed: int = 7, reps: int = 5) -> dict:
    """Forward and adjoint device times of the C3 rollout alone (the MC
    Biot-Savart step, checkpoints every ckpt steps): the forward rollout with
    the loss, and forward + backward; adjoint = the difference."""
    cfg, x, w = scenes.periodic2d(n, seed=seed, dt=0.01)
    box = VortexBox(cfg, x, mc_fraction=mc_fraction)
    dev = box.device
    w0 = torch.from_numpy(w).to(dev)
    _, _, wt = scenes.periodic2d(n, seed=target_seed, dt=0.01)
    with torch.no_grad():
        target = box.rollout(torch.from_numpy(wt).to(dev), steps, mode=FULL)

    def fwd():
        with torch.no_grad():
            return box.loss(box.rollout(w0, steps, checkpoint_every=ckpt, mode=MC), target)

    def fwd_bwd():
        wg = w0.clone().requires_grad_(True)
        box.loss(box.rollout(wg, steps, checkpoint_every=ckpt, mode=MC), target).backward()

    fwd()
    fwd_bwd()
    t_f = timed(fwd, reps)
    t_fb = timed(fwd_bwd, reps)
    return {"workload": f"periodic2d inverse problem: n={n}, {steps}-step rollout, checkpoints every {ckpt}, "
                        f"M={box.M}", "forward_ms": t_f, "forward_backward_ms": t_fb, "adjoint_ms": t_fb - t_f,
            "adjoint_over_forward": (t_fb - t_f) / t_f}


def run(n: int = 65536, steps: int = 32, ckpt: int = 8, mc_fraction: float = 1.0 / 16.0,
        Rs=(1, 4, 16, 64), opt_iters: int = 40, lr: float = 0.2, fd_coords: int = 64, seed: int = 0,
        target_seed: int = 7) -> dict:
    cfg, x, w = scenes.periodic2d(n, seed=seed, dt=0.01)
    box = VortexBox(cfg, x, mc_fraction=mc_fraction)
    dev = box.device
    w0 = torch.from_numpy(w).to(dev)
    _, _, wt = scenes.periodic2d(n, seed=target_seed, dt=0.01)
    wt = torch.from_numpy(wt).to(dev)
    out = {"workload": "periodic2d-inverse", "n": n, "M": box.M, "steps": steps, "checkpoint_every": ckpt,
           "dt": box.dt}
    with torch.no_grad():
        target = box.rollout(wt, steps, mode=FULL)
    out["target_rms_speed"] = float(target.double().pow(2).sum(1).mean().sqrt())

    # -------------------------------------------------------------- timing
    def fwd(mode=MC):
        with torch.no_grad():
            return box.loss(box.rollout(w0, steps, checkpoint_every=ckpt, mode=mode), target)

    def fwd_bwd(mode=MC):
        wg = w0.clone().requires_grad_(True)
        L = box.loss(box.rollout(wg, steps, checkpoint_every=ckpt, mode=mode), target)
        L.backward()

    fwd()
    fwd_bwd()
    t_f = timed(fwd, 5)
    t_fb = timed(fwd_bwd, 5)
    out["mc"] = {"forward_ms": t_f, "forward_backward_ms": t_fb, "adjoint_ms": t_fb - t_f,
                 "adjoint_over_forward": (t_fb - t_f) / t_f}
    t_F = timed(lambda: fwd(FULL), 2)
    t_FB = timed(lambda: fwd_bwd(FULL), 2)
    out["full_bs"] = {"forward_ms": t_F, "forward_backward_ms": t_FB, "adjoint_ms": t_FB - t_F,
                      "adjoint_over_forward": (t_FB - t_F) / t_F}
    out["mc_speedup_forward_backward"] = t_FB / t_fb
    v = box.initial_velocity(w0)
    out["plan_ms"] = timed(lambda: box.build_plan(box.x0, v, 0, MC), 5)
    plan = box.validate(box.build_plan(box.x0, v, 0, MC))
    out["n_src"], out["pairs_near"] = plan.n_src, plan.nnz
    xs = box.x0.clone().requires_grad_(True)
    ws = w0.clone().requires_grad_(True)
    g = torch.randn(n, 2, device=dev, generator=torch.Generator(device=dev).manual_seed(0))

    def op_f():
        with torch.no_grad():
            box.velocity(box.x0, w0, plan)

    def op_fb():
        u = box.velocity(xs, ws, plan)
        torch.autograd.grad((u * g).sum(), (xs, ws))

    out["op_forward_ms"] = timed(op_f, 10)
    out["op_forward_backward_ms"] = timed(op_fb, 10)
    out["op_vjp_over_forward"] = (out["op_forward_backward_ms"] - out["op_forward_ms"]) / out["op_forward_ms"]

    # ------------------------------------------------------ FD and FP32/64
    rng = np.random.default_rng(seed + 1)
    coords = rng.choice(n, fd_coords, replace=False)
    t0 = time.perf_counter()
    ad, fd = fd_check(box, w0, target.double(), coords, steps=steps, eps=1e-6, checkpoint_every=ckpt)
    out["fd"] = {"coords": fd_coords, "eps": 1e-6, "normwise_rel_err": float(np.linalg.norm(ad - fd) /
                                                                            np.linalg.norm(fd)),
                 "max_abs_err_over_max_abs_grad": float(np.max(np.abs(ad - fd)) / np.max(np.abs(fd))),
                 "seconds": time.perf_counter() - t0}
    with torch.no_grad():
        _, plans = box.rollout(w0.double(), steps, mode=MC, keep_plans=True)
    grads = {}
    for dt_ in (torch.float64, torch.float32):
        wg = w0.to(dt_).clone().requires_grad_(True)
        L = box.loss(box.rollout(wg, steps, checkpoint_every=ckpt, plans=plans, frozen=True), target)
        (grads[dt_],) = torch.autograd.grad(L, wg)
    out["fp32_vs_fp64_grad_rel"] = _nrel(grads[torch.float32].cpu(), grads[torch.float64].cpu())
    del plans

    # ------------------------------------------------------- MC vs full BS
    def grad(mode, s=None):
        wg = w0.clone().requires_grad_(True)
        L = box.loss(box.rollout(wg, steps, checkpoint_every=ckpt, mode=mode, seed=s), target)
        return torch.autograd.grad(L, wg)[0].double()

    gref = grad(FULL)
    acc = torch.zeros_like(gref)
    sweep = []
    r = 0
    for R in sorted(Rs):
        while r < R:
            acc += grad(MC, 1000 + r)
            r += 1
        m = acc / R
        sweep.append({"R": R, "rel_err": _nrel(m.cpu(), gref.cpu()), "cos": _cos(m.cpu(), gref.cpu())})
    out["mc_vs_full_grad"] = sweep

    # the other way to cut the variance: more samples in each step's plan
    # (one sampler stream, M from N/16 to N), with the cost of a gradient
    M0 = box.M
    msweep = []
    for frac in (1.0 / 16.0, 0.25, 0.5, 1.0):
        box.M = max(1, int(round(frac * n)))
        g1 = grad(MC, 3000)
        msweep.append({"M": box.M, "rel_err": _nrel(g1.cpu(), gref.cpu()), "cos": _cos(g1.cpu(), gref.cpu()),
                       "forward_backward_ms": timed(fwd_bwd, 3)})
    box.M = M0
    out["mc_grad_vs_M"] = msweep

    # ---------------------------------------------------------- inversion
    def true_loss(wv):
        with torch.no_grad():
            return float(box.loss(box.rollout(wv, steps, mode=FULL), target))

    curves = {}
    for name, mode in (("mc", MC), ("full_bs", FULL)):
        wv = w0.clone().requires_grad_(True)
        opt = torch.optim.Adam([wv], lr=lr)
        curve = [(0, true_loss(wv.detach()))]
        t0 = time.perf_counter()
        for it in range(opt_iters):
            opt.zero_grad()
            L = box.loss(box.rollout(wv, steps, checkpoint_every=ckpt, mode=mode, seed=2000 + it), target)
            L.backward()
            opt.step()
            if (it + 1) % 10 == 0 or it + 1 == opt_iters:
                curve.append((it + 1, true_loss(wv.detach())))
        torch.cuda.synchronize()
        curves[name] = {"loss": curve, "seconds_incl_evaluations": time.perf_counter() - t0}
    out["inversion"] = {"optimizer": "Adam", "lr": lr, "iterations": opt_iters, **curves}
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=65536)
    ap.add_argument("--steps", type=int, default=32)
    ap.add_argument("--opt-iters", type=int, default=40)
    ap.add_argument("--lr", type=float, default=0.2)
    ap.add_argument("--out", type=str, default=None)
    a = ap.parse_args()
    res = run(n=a.n, steps=a.steps, opt_iters=a.opt_iters, lr=a.lr)
    s = json.dumps(res)
    print(s)
    if a.out:
        with open(a.out, "w") as f:
            f.write(s + "\n")


if __name__ == "__main__":
    main()
