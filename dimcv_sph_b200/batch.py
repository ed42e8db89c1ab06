"""Scene batch: many independent channel scenes stepped together.

New form (the reference steps one scene per process).  Each scene is built by
the single-scene path (ParticleSystem + KarmanVortexSolver.initialize), so
its initial particles, boundary volumes, emitter lattice and emit interval
are the ones a lone run would have.  The scenes are concatenated into one
libdimcv context created with ``n_scenes = S``: slots carry their scene id in
``object_id``, positions stay scene-local, and ``dv_batch_step`` advances
every scene by one step (emission, activity, grid build, the substep) with
no host synchronisation, so ``capture()`` records whole steps in a CUDA graph
that ``replay()`` launches.

All scenes share the solver constants of one configuration (particle radius,
dt, density, tolerances); only the box, the obstacle, the inflow and the
sampler seed differ.  The shared cell grid is the largest scene grid; a lone
scene run with the same ``grid_num`` visits neighbours in the same order and
produces the same bits (tests/test_gpu_batch.py).
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np
import torch

from . import _lib, scenes
from ._abi import DV_SAMPLE_INVERSE_CDF, DV_SAMPLE_STRATIFIED, DvBatchScene, DvSceneState
from .fields import particle_fields, solver_fields

_SAMPLERS = {"inverse_cdf": DV_SAMPLE_INVERSE_CDF, "stratified": DV_SAMPLE_STRATIFIED}


def channel_batch_configs(n_scenes: int = 256, seed: int = 0, n_min: float = 2000, n_max: float = 60000,
                          radius: float = 0.01, dt: float = 4e-4, sampler: str = "inverse_cdf",
                          reserve_steps: int = 400):
    """Configurations of n_scenes 2-D channels (the small-channel solver
    constants: r = 0.01, h = 0.04, dt = 4e-4, M = N/16).  Fluid counts are
    log-uniform in [n_min, n_max] through the channel size (aspect 4:1,
    height sqrt(N / 10^4)), inflow U(0.5, 2), cylinder radius U(0.05, 0.15)
    (at most a quarter of the height) at (L/4, H/2).  Returns (configs,
    target fluid counts)."""
    rng = np.random.default_rng(seed)
    Ns = np.exp(rng.uniform(math.log(n_min), math.log(n_max), size=n_scenes))
    U = rng.uniform(0.5, 2.0, size=n_scenes)
    R = rng.uniform(0.05, 0.15, size=n_scenes)
    cfgs = []
    d = 2 * radius
    for s in range(n_scenes):
        H = math.sqrt(Ns[s] / 1e4)
        L = 4.0 * H
        r = min(float(R[s]), 0.25 * H)
        per = int(math.ceil(H / d))
        interval = int(math.ceil(d / (float(U[s]) * float(np.float32(dt)))))
        reserve = per * (reserve_steps // interval + 2)
        cfgs.append(scenes.channel2d(radius=radius, length=L, height=H, inflow=float(U[s]),
                                     cyl_center=(0.25 * L, 0.5 * H), cyl_radius=r, dt=dt, mc_fraction=1.0 / 16.0,
                                     sampler=sampler, seed=seed * 100003 + s, reserved=reserve))
        cfgs[-1].config["Configuration"]["computeVis"] = False
    return cfgs, Ns


def _grid_of(cfg) -> np.ndarray:
    from .params import make_params
    p = make_params(cfg)
    return np.array(list(p.grid_num)[:2])


class SceneBatch:
    def __init__(self, cfgs, device=None, capacity_margin: float = 1.0, verbose: bool = False,
                 keep_snapshots: bool = False):
        from .params import make_params
        from .particle_system import ParticleSystem
        self.cfgs = cfgs
        self.S = S = len(cfgs)
        if S < 1:
            raise ValueError("a scene batch needs at least one scene")
        self.device = torch.device(device or "cuda")
        self.lib = _lib.load()
        self.grid_num = np.max(np.stack([_grid_of(c) for c in cfgs]), axis=0)
        g0 = cfgs[0].get_cfg
        self.sampler = g0("samplerMode") or "inverse_cdf"
        if self.sampler not in _SAMPLERS:
            raise ValueError(f"scene batches sample with {sorted(_SAMPLERS)}")
        mcs = g0("mcSamples")
        self.mc_fraction = float(mcs) if mcs is not None else 1.0 / 16.0
        # per-scene initial state through the single-scene path
        snaps, counts, emit_pos, infos = [], [], [], []
        cap_total = 0
        t0 = time.perf_counter()
        for s, cfg in enumerate(cfgs):
            ps = ParticleSystem(cfg, device=self.device, grid_num=self.grid_num)
            sv = ps.build_solver()
            sv.initialize()
            cnt = ps.counters()
            n = cnt["n"]
            snaps.append({k: t[:n].clone() for k, t in ps.fields.t.items()})
            counts.append((n, cnt["n_fluid"], cnt["n_solid"]))
            off = sum(e.shape[0] for e in emit_pos)
            pos = np.zeros((0, 2), np.float32)
            em = ps.fluid_emitters[0] if ps.fluid_emitters else None
            if em is not None:
                center, size = np.array(em["squareCenter"]), np.array(em["squareSize"])
                vel = np.array(em["velocity"])
                lower = center - 0.5 * size
                cube = size + ps.particle_radius * np.abs(vel) / np.linalg.norm(vel)
                pos = ps._lattice(lower, cube)
            emit_pos.append(pos)
            infos.append({"domain_end": list(ps.domain_end), "n": n, "cap": int(ps.particle_max_num),
                          "emit_offset": off, "emit_count": pos.shape[0],
                          "emit_interval": int(sv.emit_interval) if em is not None else 0,
                          "emit_velocity": list(em["velocity"]) if em is not None else [0, 0],
                          "emit_density": float(em["density"]) if em is not None else 1000.0,
                          "emit_color": list(em.get("color", [0, 0, 0])) if em is not None else [0, 0, 0],
                          "seed": int(sv.seed), "m_V0": float(ps.m_V0)})
            cap_total += int(ps.particle_max_num)
            del sv, ps
        self.build_seconds = time.perf_counter() - t0
        self.infos = infos
        if keep_snapshots:  # the initial slots of every scene (for lone reference runs)
            self.snaps, self.snap_counts = snaps, counts
        self.cap = cap = int(cap_total * capacity_margin)
        # the batch context
        p = make_params(cfgs[0])
        for d in range(2):
            p.grid_num[d] = int(self.grid_num[d])
            p.domain_end[d] = float(max(i["domain_end"][d] for i in infos))
        p.n_scenes = S
        self.params = p
        self.stream = torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            self.ctx = self.lib.dv_create(C.byref(p), cap, C.c_void_p(self.stream.cuda_stream))
        if not self.ctx:
            raise _lib.DimcvError(f"dv_create failed: {self.lib.dv_last_error(None).decode()}")
        self._sets = [particle_fields(cap, 2, self.device), particle_fields(cap, 2, self.device)]
        self._cur = 0
        self.solver_buf = solver_fields(cap, 2, self.device)
        cur = self._sets[0]
        o = 0
        for s, snap in enumerate(snaps):
            n = counts[s][0]
            for k, t in snap.items():
                cur[k][o:o + n] = t
            cur["object_id"][o:o + n] = s
            o += n
        tot = np.sum(np.array(counts), axis=0)
        self._check(self.lib.dv_set_counts(self.ctx, int(tot[0]), int(tot[1]), int(tot[2])), "dv_set_counts")
        tab = (DvBatchScene * S)()
        for s, i in enumerate(infos):
            q = tab[s]
            for d in range(3):
                q.domain_end[d] = float(np.float32(i["domain_end"][d])) if d < 2 else 0.0
                q.emit_velocity[d] = float(np.float32(i["emit_velocity"][d])) if d < 2 else 0.0
                q.emit_color[d] = int(i["emit_color"][d])
            q.cap = i["cap"]
            q.emit_offset, q.emit_count, q.emit_interval = i["emit_offset"], i["emit_count"], i["emit_interval"]
            q.emit_density = float(np.float32(i["emit_density"]))
            q.emit_volume = float(np.float32(i["m_V0"]))
            q.seed = i["seed"]
        ep = np.ascontiguousarray(np.concatenate(emit_pos, 0) if emit_pos else np.zeros((0, 2)), np.float32)
        self._emit = ep
        self._check(self.lib.dv_batch_setup(self.ctx, tab, S, ep.ctypes.data_as(C.c_void_p) if ep.size else None,
                                            int(ep.shape[0]), float(self.mc_fraction), _SAMPLERS[self.sampler]),
                    "dv_batch_setup")
        self.steps = 0
        self.graph_steps = 0
        if verbose:
            print(f"batch of {S} scenes, {int(tot[0])} particles, capacity {cap}, grid {self.grid_num.tolist()}, "
                  f"built in {self.build_seconds:.1f} s")

    def __del__(self):
        ctx = getattr(self, "ctx", None)
        if ctx:
            try:
                self.lib.dv_destroy(ctx)
            finally:
                self.ctx = None

    def _check(self, rc, what):
        return _lib.check(self.ctx, rc, what)

    @property
    def fields(self):
        return self._sets[self._cur]

    def step(self):
        """One step of every scene (eager launches; the Jacobi loops poll)."""
        src, dst = self._sets[self._cur], self._sets[1 - self._cur]
        self._check(self.lib.dv_batch_step(self.ctx, C.byref(src.struct), C.byref(dst.struct),
                                           C.byref(self.solver_buf.struct)), "dv_batch_step")
        self._cur = 1 - self._cur
        self.steps += 1

    def capture(self, steps: int = 2):
        """Records `steps` (even) steps from the current set in a CUDA graph."""
        a, b = self._sets[self._cur], self._sets[1 - self._cur]
        self._check(self.lib.dv_batch_graph_capture(self.ctx, C.byref(a.struct), C.byref(b.struct),
                                                    C.byref(self.solver_buf.struct), int(steps)),
                    "dv_batch_graph_capture")
        self.graph_steps = int(steps)

    def replay(self):
        """Launches the captured steps (the current set is unchanged: even count)."""
        self._check(self.lib.dv_batch_graph_launch(self.ctx), "dv_batch_graph_launch")
        self.steps += self.graph_steps

    def states(self) -> list[dict]:
        out = (DvSceneState * self.S)()
        step = C.c_int64(0)
        self._check(self.lib.dv_batch_read(self.ctx, out, self.S, C.byref(step)), "dv_batch_read")
        self.device_step = step.value
        return [o.as_dict() for o in out]

    def counters(self) -> dict:
        from ._abi import DvCounters
        c = DvCounters()
        self._check(self.lib.dv_get_counters(self.ctx, C.byref(c)), "dv_get_counters")
        return c.as_dict()

    def scene_fields(self, s: int, names=("x", "v", "density", "pressure", "dfsph_factor", "material"),
                     states=None) -> dict:
        """Host copies of scene s's slots (sorted order) of the current set."""
        st = (states or self.states())[s]
        a, b = st["start"], st["end"]
        return {k: self.fields[k][a:b].cpu().numpy() for k in names}
