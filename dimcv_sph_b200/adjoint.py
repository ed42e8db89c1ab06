"""Differentiable 2-D vortex-particle rollout with hand-written adjoints.

New form (the reference has no derivatives).  One step of the rollout is

    ω̃ = Smooth(x, ω)          SPH vorticity smoothing (dimcv_sph.py:660-677)
    u  = Velocity(x, ω̃)       Monte-Carlo Biot-Savart (dimcv_sph.py:649-719),
                               without the ‖v_vort‖ < ‖v‖ gate
    x ← x + dt u               (advect, dimcv_sph.py:210-218)

with the particle vorticity ω constant along trajectories (2-D inviscid).
Smooth and Velocity are ``torch.autograd.Function``s whose forward and
backward passes are the CUDA kernels of libdimcv (``dv_vpm_*``, FP32 or
FP64); torch only gathers the particles into the plan's slot order and back.

A *plan* is built per step by the library's own pipeline on the current
positions: grid build (sort + neighbour lists), the fused ∇v sweep on the
previous step's velocity, KVN, AKDE and the stratified inverse-CDF sampler.
It freezes the neighbour lists, the samples and their weights (and, for
finite differences, the periodic image of every pair).  Gradients are the
exact derivatives of the step with the plan held fixed: the sampling pdf is
not differentiated (its parameters are treated as constants), and the
piecewise-constant structure changes only on measure-zero sets.

Positions are carried unwrapped (x + dt u, no modulo): the kernels take
minimum-image differences, and only the copy given to the grid build is
wrapped into the box.  Checkpointing keeps the state at every
``checkpoint_every``-th step and recomputes the steps in between during the
backward pass (``torch.utils.checkpoint``); plans are rebuilt bit-identically
because every kernel of the pipeline is deterministic.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import torch
from torch.utils.checkpoint import checkpoint

from . import _lib
from ._abi import DV_VPM_FULL, DV_VPM_MC, DvVpmPlan

MC = DV_VPM_MC
FULL = DV_VPM_FULL


def _prec(t: torch.Tensor) -> int:
    if t.dtype == torch.float64:
        return 64
    if t.dtype == torch.float32:
        return 32
    raise TypeError(f"unsupported dtype {t.dtype}")


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Plan:
    """Frozen structure of one step (device tensors + the dv_vpm_plan view)."""

    I32 = ("n_src", "perm", "inv_perm", "nbr_off", "nbr", "src", "slot_src")
    F32 = ("src_a", "slot_a", "f", "m_V")

    def __init__(self, n: int, src_cap: int, nbr_cap: int, device=None, buffers=None):
        self.n, self.src_cap, self.nbr_cap = n, src_cap, nbr_cap
        isz = {"n_src": 1, "perm": n, "inv_perm": n, "nbr_off": n + 1, "nbr": nbr_cap, "src": src_cap,
               "slot_src": n}
        fsz = {"src_a": src_cap, "slot_a": n, "f": n, "m_V": n}
        if buffers is None:
            buffers = (torch.empty(sum(isz.values()), dtype=torch.int32, device=device),
                       torch.empty(sum(fsz.values()), dtype=torch.float32, device=device))
        self._i32, self._f32 = buffers
        self.t = {}
        for buf, sizes in ((self._i32, isz), (self._f32, fsz)):
            o = 0
            for k, m in sizes.items():
                self.t[k] = buf[o:o + m]
                o += m
        self.xbar = None  # nominal slot-order positions (set when the plan is kept)
        self.n_src = None
        self.nnz = None

    def buffers(self):
        return self._i32, self._f32

    def meta(self):
        return self.n, self.src_cap, self.nbr_cap

    @property
    def perm(self):
        return self.t["perm"]

    @property
    def inv_perm(self):
        return self.t["inv_perm"]

    def struct(self, xbar: torch.Tensor | None = None) -> DvVpmPlan:
        s = DvVpmPlan()
        s.n, s.src_cap, s.nbr_cap = self.n, self.src_cap, self.nbr_cap
        for k in self.I32 + self.F32:
            setattr(s, k, self.t[k].data_ptr())
        s.xbar = xbar.data_ptr() if xbar is not None else None
        return s


def _save(ctx, box, plan, xbar, *ts):
    """Saves the plan through save_for_backward, so that checkpointing drops
    and recomputes it with the other saved tensors."""
    i32, f32 = plan.buffers()
    extra = (xbar,) if xbar is not None else ()
    ctx.save_for_backward(i32, f32, *ts, *extra)
    ctx.box, ctx.meta, ctx.nts, ctx.has_xbar = box, plan.meta(), len(ts), xbar is not None


def _load(ctx):
    saved = ctx.saved_tensors
    i32, f32 = saved[0], saved[1]
    ts = saved[2:2 + ctx.nts]
    xbar = saved[2 + ctx.nts] if ctx.has_xbar else None
    n, src_cap, nbr_cap = ctx.meta
    return ctx.box, Plan(n, src_cap, nbr_cap, buffers=(i32, f32)), xbar, ts


class _Smooth(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xs, ws, box, plan, xbar):
        out = torch.empty_like(ws)
        st = plan.struct(xbar)
        box._check(box.lib.dv_vpm_smooth(box.ctx, C.byref(st), _prec(xs), _ptr(xs), _ptr(ws), _ptr(out)),
                   "dv_vpm_smooth")
        _save(ctx, box, plan, xbar, xs, ws)
        return out

    @staticmethod
    def backward(ctx, g):
        box, plan, xbar, (xs, ws) = _load(ctx)
        g = g.contiguous()
        gw = torch.empty_like(ws)
        gx = torch.empty_like(xs)
        st = plan.struct(xbar)
        box._check(box.lib.dv_vpm_smooth_bwd(box.ctx, C.byref(st), _prec(xs), _ptr(xs), _ptr(ws), _ptr(g),
                                             _ptr(gw), _ptr(gx)), "dv_vpm_smooth_bwd")
        return gx, gw, None, None, None


class _Curl(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xs, vs, box, plan, xbar):
        out = torch.empty(xs.shape[0], dtype=xs.dtype, device=xs.device)
        st = plan.struct(xbar)
        box._check(box.lib.dv_vpm_curl(box.ctx, C.byref(st), _prec(xs), _ptr(xs), _ptr(vs), _ptr(out)),
                   "dv_vpm_curl")
        _save(ctx, box, plan, xbar, xs, vs)
        return out

    @staticmethod
    def backward(ctx, g):
        box, plan, xbar, (xs, vs) = _load(ctx)
        g = g.contiguous()
        gv = torch.empty_like(vs)
        gx = torch.empty_like(xs)
        st = plan.struct(xbar)
        box._check(box.lib.dv_vpm_curl_bwd(box.ctx, C.byref(st), _prec(xs), _ptr(xs), _ptr(vs), _ptr(g),
                                           _ptr(gv), _ptr(gx)), "dv_vpm_curl_bwd")
        return gx, gv, None, None, None


class _Velocity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xs, wt, box, plan, xbar):
        u = torch.empty_like(xs)
        ws, nb = box._workspace(plan, _prec(xs))
        st = plan.struct(xbar)
        box._check(box.lib.dv_vpm_velocity(box.ctx, C.byref(st), _prec(xs), _ptr(xs), _ptr(wt), _ptr(u),
                                           _ptr(ws), nb), "dv_vpm_velocity")
        _save(ctx, box, plan, xbar, xs, wt)
        return u

    @staticmethod
    def backward(ctx, g):
        box, plan, xbar, (xs, wt) = _load(ctx)
        g = g.contiguous()
        gw = torch.empty_like(wt)
        gx = torch.empty_like(xs)
        ws, nb = box._workspace(plan, _prec(xs))
        st = plan.struct(xbar)
        box._check(box.lib.dv_vpm_velocity_bwd(box.ctx, C.byref(st), _prec(xs), _ptr(xs), _ptr(wt), _ptr(g),
                                               _ptr(gw), _ptr(gx), _ptr(ws), nb), "dv_vpm_velocity_bwd")
        return gx, gw, None, None, None


class VortexBox:
    """N vortex particles on a periodic 2-D box (a ParticleSystem whose
    particles are all fluid), with the differentiable rollout."""

    def __init__(self, cfg, x0: np.ndarray, device=None, mc_fraction: float = 1.0 / 16.0):
        from .dimcv_sph import DIMCVSPHSolver
        from .particle_system import ParticleSystem
        n = int(x0.shape[0])
        self.n = n
        self.ps = ParticleSystem(cfg, device=device, capacity=n)
        if self.ps.dim != 2 or not self.ps.params.periodic:
            raise ValueError("VortexBox needs a 2-D periodic configuration")
        self.device = self.ps.device
        self.lib, self.ctx = self.ps.lib, self.ps.ctx
        x0 = np.ascontiguousarray(x0, dtype=np.float32)
        z = np.zeros(n)
        self.ps.add_particles(0, n, x0, np.zeros_like(x0), np.full(n, 1000.0), z, np.ones(n, np.int32),
                              np.ones(n, np.int32), np.zeros((n, 3), np.int32))
        self.solver = DIMCVSPHSolver(self.ps)
        self.solver.sampler = "stratified"
        self.solver.initialize()
        self.x0 = torch.from_numpy(x0).to(self.device)
        self.box = torch.tensor(list(self.ps.params.box)[:2], dtype=torch.float64, device=self.device)
        self.start = torch.tensor(list(self.ps.params.domain_start)[:2], dtype=torch.float64, device=self.device)
        self.dt = float(self.ps.params.dt)
        self.M = max(1, int(round(mc_fraction * n)))
        self.seed = self.solver.seed
        self.nbr_cap = n * 24
        self._ws = {}

    # ----------------------------------------------------------- plumbing
    def _check(self, rc, what):
        return _lib.check(self.ctx, rc, what)

    def _workspace(self, plan: Plan, prec: int):
        key = (plan.n, plan.src_cap, prec)
        if key not in self._ws:
            nb = int(self.lib.dv_vpm_workspace_bytes(self.ctx, plan.n, plan.src_cap, prec))
            self._check(nb, "dv_vpm_workspace_bytes")
            self._ws[key] = torch.empty(max(nb, 1), dtype=torch.uint8, device=self.device)
        ws = self._ws[key]
        return ws, ws.numel()

    def wrap(self, x: torch.Tensor) -> torch.Tensor:
        """Positions folded into [start, start + box) as float32 (for the grid)."""
        xd = x.detach().double()
        y = self.start + torch.remainder(xd - self.start, self.box)
        y = y.float()
        hi = (self.start + self.box).float()
        return torch.where(y >= hi, self.start.float().expand_as(y), y)

    # ---------------------------------------------------------------- plan
    def build_plan(self, x: torch.Tensor, v: torch.Tensor | None, step: int, mode: int = MC,
                   seed: int | None = None) -> Plan:
        """Plan of one step at positions x (caller order) with v (caller
        order, float32) as the velocity whose KVN sets the sampling pdf."""
        n, ps, sv = self.n, self.ps, self.solver
        ps.x[:n] = self.wrap(x)
        if v is not None:
            ps.v[:n] = v.detach().float()
        ps.initialize_particle_system()  # sort + neighbour lists
        if mode == MC:
            sv.rng_step = int(step)
            sv.seed = int(self.seed if seed is None else seed)
            sv.init()                                  # ∇v of v
            sv.compute_kinematic_vorticity_num_sample()  # KVN
            sv.compute_kernel_density()                # AKDE, FP64 kden_sum
            sv._calls("dv_sample", 3, sv.seed, sv.rng_step, self.M)  # stratified inverse-CDF draws
            src_cap = self.M
        else:
            src_cap = n
        plan = Plan(n, src_cap, self.nbr_cap, self.device)
        st = plan.struct()
        self._check(self.lib.dv_vpm_plan_build(self.ctx, C.byref(ps.fields_struct), C.byref(ps.solver_buf.struct),
                                               mode, C.byref(st)), "dv_vpm_plan_build")
        return plan

    def validate(self, plan: Plan):
        """Reads the plan's source and pair counts (synchronises)."""
        ns = int(plan.t["n_src"][0].item())
        if ns < 0:
            raise _lib.DimcvError("dv_vpm_plan_build failed (count mismatch, missing lists or capacity)")
        plan.n_src = ns
        plan.nnz = int(plan.t["nbr_off"][plan.n].item())
        return plan

    # ---------------------------------------------------------------- step
    def velocity(self, x: torch.Tensor, w: torch.Tensor, plan: Plan, frozen: bool = False) -> torch.Tensor:
        """u (caller order) from positions x [n,2] and vorticity w [n]."""
        xs = x.index_select(0, plan.perm)
        ws = w.index_select(0, plan.perm)
        xbar = None
        if frozen:
            if plan.xbar is None:
                raise ValueError("frozen images need a plan kept from a nominal rollout")
            xbar = plan.xbar.to(xs.dtype).contiguous()
        wt = _Smooth.apply(xs, ws, self, plan, xbar)
        us = _Velocity.apply(xs, wt, self, plan, xbar)
        if plan.xbar is None and getattr(plan, "keep", False):
            plan.xbar = xs.detach().clone()
        return us.index_select(0, plan.inv_perm)

    def curl(self, x: torch.Tensor, v: torch.Tensor, plan: Plan, frozen: bool = False) -> torch.Tensor:
        """SPH vorticity ω (caller order) of velocities v [n,2] at positions x
        (compute_vorticity, dimcv_sph.py:228-248), differentiable in x and v."""
        xs = x.index_select(0, plan.perm)
        vs = v.index_select(0, plan.perm).contiguous()
        xbar = plan.xbar.to(xs.dtype).contiguous() if frozen else None
        ws = _Curl.apply(xs, vs, self, plan, xbar)
        return ws.index_select(0, plan.inv_perm)

    def initial_velocity(self, w: torch.Tensor) -> torch.Tensor:
        """Full Biot-Savart velocity of the initial state (float32, no
        gradient): the velocity whose KVN sets the first step's pdf."""
        with torch.no_grad():
            plan = self.build_plan(self.x0, None, 0, FULL)
            return self.velocity(self.x0, w.detach().float(), plan).float()

    def _segment(self, x, w, v, k0: int, k1: int, mode: int, plans, frozen: bool, keep: list | None,
                 seed: int | None = None):
        for k in range(k0, k1):
            if plans is not None:
                plan = plans[k]
            else:
                plan = self.build_plan(x, v, k, mode, seed)
                if keep is not None:
                    plan.keep = True
                    keep.append(plan)
            u = self.velocity(x, w, plan, frozen)
            v = u.detach().float()
            x = x + self.dt * u
        return x, v

    def rollout(self, w0: torch.Tensor, steps: int = 32, checkpoint_every: int | None = 8, mode: int = MC,
                plans: list | None = None, frozen: bool = False, keep_plans: bool = False, v0=None,
                seed: int | None = None):
        """Final velocity u_K (caller order) after `steps` advection steps
        from the fixed initial positions; dtype of w0.  With keep_plans the
        plans (and their nominal positions) are returned for reuse.  `seed`
        selects the sampler stream (default: the configuration's seed)."""
        if seed is None:
            seed = self.seed
        dtype = w0.dtype
        x = self.x0.to(dtype)
        v = v0 if v0 is not None else (None if plans is not None else self.initial_velocity(w0))
        keep = [] if keep_plans else None
        use_ckpt = checkpoint_every and torch.is_grad_enabled() and w0.requires_grad and not keep_plans
        k = 0
        while k < steps:
            k1 = min(steps, k + (checkpoint_every or steps))
            if use_ckpt:
                x, v = checkpoint(self._segment, x, w0, v, k, k1, mode, plans, frozen, None, seed,
                                  use_reentrant=False, preserve_rng_state=False)
            else:
                x, v = self._segment(x, w0, v, k, k1, mode, plans, frozen, keep, seed)
            k = k1
        if plans is not None:
            plan = plans[steps]
        else:
            plan = self.build_plan(x, v, steps, mode, seed)
            if keep is not None:
                plan.keep = True
                keep.append(plan)
        u = self.velocity(x, w0, plan, frozen)
        return (u, keep) if keep_plans else u

    @staticmethod
    def loss(u: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
        d = u - target.to(u.dtype)
        return (d * d).sum() / u.shape[0]


def fd_check(box: VortexBox, w0: torch.Tensor, target: torch.Tensor, coords: np.ndarray, steps: int = 32,
             eps: float = 1e-6, mode: int = MC, checkpoint_every: int | None = 8):
    """FP64 adjoint gradient of the rollout loss vs FP64 central differences
    on the given vorticity coordinates, with the nominal plans and periodic
    images frozen.  Returns (adjoint [len(coords)], fd [len(coords)])."""
    w = w0.detach().double()
    with torch.no_grad():
        _, plans = box.rollout(w, steps, mode=mode, keep_plans=True)
    for p in plans:
        box.validate(p)
    wg = w.clone().requires_grad_(True)
    L = VortexBox.loss(box.rollout(wg, steps, checkpoint_every=checkpoint_every, mode=mode, plans=plans,
                                   frozen=True), target)
    (g,) = torch.autograd.grad(L, wg)
    ad = g[torch.as_tensor(coords, device=g.device)].cpu().numpy()
    fd = np.zeros(len(coords))
    with torch.no_grad():
        for t, c in enumerate(coords):
            wp = w.clone()
            wp[int(c)] += eps
            lp = VortexBox.loss(box.rollout(wp, steps, mode=mode, plans=plans, frozen=True), target)
            wm = w.clone()
            wm[int(c)] -= eps
            lm = VortexBox.loss(box.rollout(wm, steps, mode=mode, plans=plans, frozen=True), target)
            fd[t] = (lp.item() - lm.item()) / (2 * eps)
    return ad, fd


def timed(fn, reps: int = 3):
    """Median device time (ms) of fn() over reps runs, CUDA events."""
    ts = []
    for _ in range(reps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))
