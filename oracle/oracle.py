"""ctypes driver of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Mirrors the operator sequence of dimcv_sph_b200 on numpy copies of the
particle state so tests can run both on identical inputs.  Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline use it, as the checker.
The oracle restates the reference (Haok-Z/DIMCV-SPH) kernels in C++; see
dimcv_oracle.cpp for the cited lines.  Parity with the reference itself is
unpinned (no reference tests or fixtures exist; Taichi is not installed).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

from dimcv_sph_b200._abi import (PARTICLE_FIELDS, SOLVER_FIELDS, DvCounters, DvFields, DvParams,
                                 DvSolverFields, components, make_struct)

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libdimcv_oracle.so"
_NP = {"f32": np.float32, "i32": np.int32, "u8": np.uint8}

_lib = None


def build():
    r = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        P, FP, SP = C.c_void_p, C.POINTER(DvFields), C.POINTER(DvSolverFields)
        sig = {
            "dvo_create": (P, [C.POINTER(DvParams), C.c_int64, C.c_int]),
            "dvo_destroy": (None, [P]),
            "dvo_set_counts": (None, [P, C.c_int, C.c_int, C.c_int]),
            "dvo_get_counters": (None, [P, C.POINTER(DvCounters)]),
            "dvo_set_num_samples": (None, [P, C.c_int]),
            "dvo_set_counters": (None, [P, C.POINTER(DvCounters)]),
            "dvo_set_sample": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int]),
            "dvo_add_particles": (C.c_int, [P, FP, P, P, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int,
                                            C.c_int, C.c_int, C.c_int, C.c_int, C.c_float]),
            "dvo_update_activity": (C.c_int, [P, FP]),
            "dvo_grid_build": (C.c_int, [P, FP, FP]),
            "dvo_get_permutation": (C.c_int, [P, P]),
            "dvo_neighbor_lists": (C.c_int64, [P, FP, P, P, C.c_int64]),
            "dvo_density_error": (C.c_double, [P, FP, C.c_float]),
            "dvo_scale_factor": (C.c_int, [P, FP, C.c_float]),
            "dvo_divergence_solve": (C.c_int, [P, FP, P]),
            "dvo_pressure_solve": (C.c_int, [P, FP, P]),
            "dvo_kvn_sample": (C.c_int, [P, FP, SP, C.c_uint64, C.c_uint64, C.c_int]),
            "dvo_sample": (C.c_int, [P, FP, SP, C.c_int, C.c_uint64, C.c_uint64, C.c_int]),
            "dvo_vvpe_mc": (C.c_int, [P, FP, SP, C.c_int]),
            "dvo_bs_full": (C.c_int, [P, FP, P, P, C.c_int, P]),
            "dvo_enforce_boundary": (C.c_int, [P, FP, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
            "dvo_set_dynamic_rigid": (None, [P, C.c_int]),
        }
        for name in ("dvo_boundary_volume", "dvo_densities", "dvo_dfsph_factor", "dvo_density_change",
                     "dvo_density_adv", "dvo_divergence_iteration", "dvo_pressure_iteration",
                     "dvo_nonpressure", "dvo_predict_velocity", "dvo_advect", "dvo_life_time",
                     "dvo_moving_boundary_volume"):
            sig[name] = (C.c_int, [P, FP])
        for name in ("dvo_dimcv_vorticity", "dvo_d_vorticity", "dvo_smooth_d_vort", "dvo_record_samples",
                     "dvo_akde", "dvo_vis"):
            sig[name] = (C.c_int, [P, FP, SP])
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class NpFields:
    def __init__(self, spec, struct_cls, capacity, dim):
        self.a = {}
        for name, (dt, comp) in spec.items():
            k = components(comp, dim)
            self.a[name] = np.zeros((capacity,) if k == 1 else (capacity, k), dtype=_NP[dt])
        self.struct = make_struct(struct_cls, {n: v.ctypes.data for n, v in self.a.items()})

    def __getitem__(self, k):
        return self.a[k]


class OracleSim:
    """Oracle state + operators.  order_mode 0 visits neighbours in the CUDA
    library's Morton order, 1 in the reference's row-major order."""

    def __init__(self, params: DvParams, capacity: int, order_mode: int = 0):
        self.lib = load()
        self.params = params
        self.dim = params.dim
        self.capacity = capacity
        self.ctx = self.lib.dvo_create(C.byref(params), capacity, order_mode)
        self.sets = [NpFields(PARTICLE_FIELDS, DvFields, capacity, self.dim),
                     NpFields(PARTICLE_FIELDS, DvFields, capacity, self.dim)]
        self.cur = 0
        self.solver = NpFields(SOLVER_FIELDS, DvSolverFields, capacity, self.dim)

    def __del__(self):
        if getattr(self, "ctx", None):
            self.lib.dvo_destroy(self.ctx)
            self.ctx = None

    @property
    def f(self) -> NpFields:
        return self.sets[self.cur]

    def _fp(self):
        return C.byref(self.f.struct)

    def _sp(self):
        return C.byref(self.solver.struct)

    def load_snapshot(self, snap: dict, counters: dict):
        """Copies a ParticleSystem.snapshot() (first n slots) into the oracle."""
        n = counters["n"]
        for k, v in snap.items():
            if k.startswith("solver."):
                self.solver.a[k[7:]][:n] = v
            else:
                self.f.a[k][:n] = v
        c = DvCounters()
        for k, _ in DvCounters._fields_:
            if k in counters:
                setattr(c, k, counters[k])
        self.lib.dvo_set_counters(self.ctx, C.byref(c))

    def counters(self) -> dict:
        c = DvCounters()
        self.lib.dvo_get_counters(self.ctx, C.byref(c))
        return c.as_dict()

    def snapshot(self) -> dict:
        n = self.counters()["n"]
        out = {k: v[:n].copy() for k, v in self.f.a.items()}
        out.update({"solver." + k: v[:n].copy() for k, v in self.solver.a.items()})
        return out

    # operators (names follow the reference methods)
    def update_activity(self):
        self.lib.dvo_update_activity(self.ctx, self._fp())

    def counting_sort(self):
        src, dst = self.sets[self.cur], self.sets[1 - self.cur]
        self.lib.dvo_grid_build(self.ctx, C.byref(src.struct), C.byref(dst.struct))
        self.cur = 1 - self.cur

    def initialize_particle_system(self):
        self.update_activity()
        self.counting_sort()

    def permutation(self):
        n = self.counters()["n"]
        out = np.zeros(max(n, 1), dtype=np.int32)
        self.lib.dvo_get_permutation(self.ctx, out.ctypes.data)
        return out[:n]

    def neighbor_lists(self):
        n = self.counters()["n"]
        off = np.zeros(n + 1, dtype=np.int64)
        total = self.lib.dvo_neighbor_lists(self.ctx, self._fp(), off.ctypes.data, None, 0)
        nbr = np.zeros(max(total, 1), dtype=np.int32)
        self.lib.dvo_neighbor_lists(self.ctx, self._fp(), off.ctypes.data, nbr.ctypes.data, total)
        return off, nbr[:total]

    def call(self, name, *args):
        return getattr(self.lib, "dvo_" + name)(self.ctx, self._fp(), *args)

    def calls(self, name, *args):
        return getattr(self.lib, "dvo_" + name)(self.ctx, self._fp(), self._sp(), *args)

    def add_particles(self, pos, vel, object_id, density, pressure, material, is_dynamic, color, m_V0):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        vel = np.ascontiguousarray(vel, dtype=np.float32)
        self.lib.dvo_add_particles(self.ctx, self._fp(), pos.ctypes.data, vel.ctypes.data, pos.shape[0],
                                   object_id, density, pressure, material, is_dynamic, *color, m_V0)

    def divergence_solve(self):
        it = C.c_int(0)
        self.lib.dvo_divergence_solve(self.ctx, self._fp(), C.addressof(it))
        return it.value

    def pressure_solve(self):
        it = C.c_int(0)
        self.lib.dvo_pressure_solve(self.ctx, self._fp(), C.addressof(it))
        return it.value

    def bs_full(self, omega: np.ndarray, targets: np.ndarray | None, nt: int) -> np.ndarray:
        om = np.ascontiguousarray(omega, dtype=np.float32)
        out = np.zeros((nt, 4), dtype=np.float64)
        tp = None
        if targets is not None:
            targets = np.ascontiguousarray(targets, dtype=np.int32)
            tp = targets.ctypes.data
        self.lib.dvo_bs_full(self.ctx, self._fp(), om.ctypes.data, tp, nt, out.ctypes.data)
        return out

    def substep(self, seed=0, step=0, sampler="bernoulli", M=0, compute_vis=True, vvpe_precision=32):
        """KarmanVortexSolver.substep (karman_vortex.py:232-242) on the oracle."""
        self.call("densities")
        self.call("dfsph_factor")
        it_div = self.divergence_solve()
        self.call("nonpressure")
        self.calls("dimcv_vorticity")
        self.calls("d_vorticity")
        self.calls("smooth_d_vort")
        self.calls("kvn_sample", seed, step, 1 if sampler == "bernoulli" else 0)
        if sampler == "bernoulli":
            self.calls("record_samples")
        self.calls("akde")
        if sampler == "inverse_cdf":
            self.calls("sample", 1, seed, step, M)
        elif sampler == "injected":
            self.lib.dvo_set_num_samples(self.ctx, M)
        self.calls("vvpe_mc", vvpe_precision)
        self.call("life_time")
        self.call("predict_velocity")
        it_p = self.pressure_solve()
        if compute_vis:
            self.calls("vis")
        self.call("advect")
        return it_div, it_p
