"""SPHBase / DIMCVSPHSolver with the reference's method names
(sph_base.py:5-232, dimcv_sph.py:6-819); every method is one or a few
libdimcv calls on the particle system's current field set.

Sampling (new options, defaults = reference):
  samplerMode  "bernoulli" (dimcv_sph.py:305-335, Philox in place of the
               time-seeded ti.random), "inverse_cdf" (M draws from the FP64
               AKDE CDF) or "injected" (the caller fills sample_idx);
  mcSamples    M for inverse_cdf as an int, or a fraction of the fluid count;
  seed         RNG seed (default 0).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._abi import (DV_SAMPLE_BERNOULLI, DV_SAMPLE_INJECTED, DV_SAMPLE_INVERSE_CDF, DV_SAMPLE_STRATIFIED,
                   DV_SOLVE_NONPRESSURE, DV_SOLVE_PREPARED, DV_SOLVE_VIS)
from .particle_system import Scalar

_MODES = {"bernoulli": DV_SAMPLE_BERNOULLI, "inverse_cdf": DV_SAMPLE_INVERSE_CDF,
          "injected": DV_SAMPLE_INJECTED, "stratified": DV_SAMPLE_STRATIFIED}


class SPHBase:
    def __init__(self, particle_system):
        self.ps = particle_system
        self.lib = self.ps.lib
        self.ctx = self.ps.ctx
        g = self.ps.cfg.get_cfg
        self.g = np.array(g("gravitation"))
        self.viscosity = 1e-3
        self.density_0 = g("density0") if g("density0") is not None else 1000.0
        self._dt = float(np.float32(g("timeStepSize") if g("timeStepSize") is not None else 1e-4))
        self.dt = Scalar(lambda: self._dt, self._set_dt)

    def _set_dt(self, value):
        # the reference keeps inv_dt / inv_dt2 from construction time
        # (dimcv_sph.py:27-28); only dt itself changes here too
        self._dt = float(np.float32(value))
        self.ps.params.dt = self._dt
        _lib.check(self.ctx, self.lib.dv_set_params(self.ctx, C.byref(self.ps.params)), "dv_set_params")

    def _call(self, name, *args):
        fn = getattr(self.lib, name)
        return _lib.check(self.ctx, fn(self.ctx, C.byref(self.ps.fields_struct), *args), name)

    def _calls(self, name, *args):
        fn = getattr(self.lib, name)
        return _lib.check(self.ctx, fn(self.ctx, C.byref(self.ps.fields_struct),
                                       C.byref(self.ps.solver_buf.struct), *args), name)

    def initialize(self):  # sph_base.py:80-85
        self.ps.initialize_particle_system()
        self.compute_static_boundary_volume()
        self.compute_moving_boundary_volume()

    def compute_static_boundary_volume(self):  # sph_base.py:91-98
        self._call("dv_boundary_volume")

    def compute_moving_boundary_volume(self):  # sph_base.py:105-112
        if getattr(self.ps, "has_dynamic_rigid", False):
            self._call("dv_moving_boundary_volume")

    def substep(self):
        pass

    def enforce_boundary_3D(self, particle_type: int):  # sph_base.py:118-179
        """Clamps the dynamic particles of this material into
        [padding, domain_size - padding] per axis (bounds in f32, as the
        reference's kernel constants) and reflects their velocity with loss."""
        ps = self.ps
        pad = np.float32(ps.padding)
        lo = (C.c_float * 3)(*([float(pad)] * 3))
        hi = (C.c_float * 3)(*[float(np.float32(np.float32(ps.domain_size[d]) - pad)) if d < ps.dim else 0.0
                               for d in range(3)])
        self._call("dv_enforce_boundary", int(particle_type), lo, hi)

    enforce_boundary_2D = enforce_boundary_3D

    def step(self):  # sph_base.py:224-232
        self.ps.initialize_particle_system()
        self.compute_moving_boundary_volume()
        self.substep()
        if self.ps.cfg.get_cfg("bounceBackBoundary"):
            if self.ps.dim == 2:
                self.enforce_boundary_2D(self.ps.material_fluid)
            else:
                self.enforce_boundary_3D(self.ps.material_fluid)


class DIMCVSPHSolver(SPHBase):
    def __init__(self, particle_system):
        super().__init__(particle_system)
        g = self.ps.cfg.get_cfg
        self.surface_tension = 0
        self.eps = 1e-6
        self.inv_eps = 1.0 / self.eps
        self.volume_scale = g("volumeScale")
        if self.volume_scale is not None:
            self.vp_volume = self.volume_scale * self.ps.m_V0
        self.m_max_iterations_v = int(g("maxIterationsV") or 100)
        self.m_max_iterations = int(g("maxIterations") or 100)
        self.m_eps = 1e-5
        self.max_error_V = 0.1
        self.max_error = 0.05
        self.inv_dt = 1.0 / self._dt
        self.inv_dt2 = 1.0 / (self._dt * self._dt)
        self.vortex_enforcing_domain_start = g("vortexEnforcingDomainStart")
        self.vortex_enforcing_domain_end = g("vortexEnforcingDomainEnd")
        self.a = g("GenProbPara")
        self.b = g("DelProbPara")
        self.divergence_transit_area = g("divergenceTransitArea")
        self.sampler = g("samplerMode") or "bernoulli"
        if self.sampler not in _MODES:
            raise ValueError(f"samplerMode must be one of {sorted(_MODES)}")
        self.mc_samples = g("mcSamples")
        self.seed = int(g("seed") or 0)
        self.rng_step = 0
        self.injected_num_samples = 0
        self.last_iters = (0, 0)
        # emitter interval (dimcv_sph.py:66-74)
        self.cnt = 0
        self.emit_interval = 1
        for emitter in self.ps.fluid_emitters:
            init_v = np.array(emitter["velocity"])
            self.emit_interval = int(np.ceil(self.ps.particle_diameter / (np.linalg.norm(init_v) * self._dt)))
            break
        sb = self.ps.solver_buf
        self.num_samples = Scalar(lambda: self.ps.counters()["num_samples"], self._set_num_samples)
        self.kden_sum = Scalar(lambda: self.ps.counters()["kden_sum_f32"])
        self._sb = sb

    # solver fields (index-stable; views of the padded buffers)
    d_vort = property(lambda self: self._sb["d_vort"][:, :3])
    d_vort_smoothed = property(lambda self: self._sb["d_vort_smoothed"][:, :3])
    v_star = property(lambda self: self._sb["v_star"][:, : self.ps.dim])
    grad_v = property(lambda self: self._sb["grad_v"].view(-1, self.ps.dim, self.ps.dim))
    x_temp = property(lambda self: self._sb["x_temp"][:, : self.ps.dim])
    sample_idx = property(lambda self: self._sb["sample_idx"])
    kinematic_vort_num = property(lambda self: self._sb["kvn"])
    kernel_density = property(lambda self: self._sb["kden"])
    v_vort = property(lambda self: self._sb["v_vort"][:, :3])
    vorticity_vis = property(lambda self: self._sb["vorticity_vis"][:, :3])

    def _set_num_samples(self, value):
        self.injected_num_samples = int(value)
        self._calls("dv_sample", DV_SAMPLE_INJECTED, 0, 0, int(value))

    # ----------------------------------------------------------- DFSPH
    # Sweeps that the reference runs back to back over the same neighbours
    # are fused (dv_densities_factor_change, the divergence solve's residual
    # sweep with the non-pressure forces, the pressure solve's opening sweep
    # with the vis sweep, dv_vorticity_dvort): the first
    # method computes all the results and a later one skips its sweep while
    # nothing it reads can have changed: no library kernel has run since
    # (the context's launch count) and no tensor it reads was written in place
    # by torch (the tensors' version counters, which views share).
    # compute_densities thereby also writes density_adv, which the reference
    # reads only after divergence_solve's own compute_density_change.
    _FACTOR_READS = ("x", "m", "m_V", "material")          # compute_DFSPH_factor
    _CHANGE_READS = ("x", "v", "m_V", "material")          # compute_density_change
    _DVORT_READS = ("x", "m_V", "material", "vorticity")   # compute_d_vorticity, with v_star
    _NONPRESSURE_READS = ("x", "v", "m_V", "material", "is_dynamic")  # compute_non_pressure_forces
    _VIS_READS = ("x", "m_V", "material", "vorticity")     # copy_x_temp + compute_vorticity_vis
    _fused_densities = None
    _fused_nonpressure = None
    _fused_vis = None
    _fused_dvort = None

    def _launches(self):
        return self.lib.dv_launch_count(self.ctx)

    def _fusion_mark(self, names, solver_names=()):
        f, sb = self.ps.fields, self._sb
        return {"at": self._launches(), "set": f,
                "ver": {**{n: f[n]._version for n in names}, **{"sb." + n: sb[n]._version for n in solver_names}}}

    def _fusion_fresh(self, mark, names, solver_names=()) -> bool:
        if mark is None or mark["at"] != self._launches() or mark["set"] is not self.ps.fields:
            return False
        f, sb, ver = self.ps.fields, self._sb, mark["ver"]
        return all(f[n]._version == ver[n] for n in names) and \
            all(sb[n]._version == ver["sb." + n] for n in solver_names)

    def compute_DFSPH_factor(self):  # dimcv_sph.py:86-106
        if self._fusion_fresh(self._fused_densities, self._FACTOR_READS):
            return  # computed by compute_densities' sweep, bit-identical
        self._call("dv_dfsph_factor")

    def compute_densities(self):  # :139-148 (with :86-106 and :337-358 in the same sweep)
        self._call("dv_densities_factor_change")
        self._fused_densities = self._fusion_mark(set(self._FACTOR_READS) | set(self._CHANGE_READS))

    def compute_non_pressure_forces(self):  # :195-208
        if self._fusion_fresh(self._fused_nonpressure, self._NONPRESSURE_READS):
            return  # computed by divergence_solve's last residual sweep, bit-identical
        self._call("dv_nonpressure")

    def advect(self):  # :210-218
        self._call("dv_advect")

    def predict_velocity(self):  # :220-226
        self._call("dv_predict_velocity")

    def compute_density_change(self):  # :337-358
        if self._fusion_fresh(self._fused_densities, self._CHANGE_READS):
            return  # computed by compute_densities' sweep, bit-identical
        self._call("dv_density_change")

    def multiply_time_step(self, field, time_step):  # :395-399
        if field is not None and field is not self.ps.dfsph_factor and \
                field.data_ptr() != self.ps.dfsph_factor.data_ptr():
            raise ValueError("multiply_time_step is defined for ps.dfsph_factor only")
        self._call("dv_scale_factor", float(np.float32(time_step)))

    def compute_density_error(self, offset):  # :407-419 (FP64 sum)
        out = C.c_double()
        self._call("dv_density_error", float(np.float32(offset)), C.byref(out))
        return out.value

    def divergence_solver_iteration_kernel(self):  # :421-443
        self._call("dv_divergence_iteration")

    def compute_density_adv(self):  # :470-479
        self._call("dv_density_adv")

    def pressure_solve_iteration_kernel(self):  # :495-508
        self._call("dv_pressure_iteration")

    def pressure_solve_iteration(self):  # :585-589
        self.pressure_solve_iteration_kernel()
        self.compute_density_adv()
        return self.compute_density_error(self.density_0) / self.ps.fluid_particle_num[None]

    def divergence_solver_iteration(self):  # :591-595
        self.divergence_solver_iteration_kernel()
        self.compute_density_change()
        return self.compute_density_error(0.0) / self.ps.fluid_particle_num[None]

    def divergence_solve(self):
        """dimcv_sph.py:376-393, with the Jacobi loop on the device."""
        it = C.c_int32(0)
        flags = DV_SOLVE_NONPRESSURE
        if self._fusion_fresh(self._fused_densities, self._CHANGE_READS):
            flags |= DV_SOLVE_PREPARED
        self._call("dv_divergence_solve_ex", flags, C.byref(it) if self.track_iterations else None)
        self._fused_nonpressure = self._fusion_mark(self._NONPRESSURE_READS)
        self.last_iters = (it.value, self.last_iters[1])

    def pressure_solve(self):
        """dimcv_sph.py:597-614, with the Jacobi loop on the device; when the
        substep draws the vis fields, its opening sweep computes them too."""
        it = C.c_int32(0)
        flags = DV_SOLVE_VIS if self.compute_vis else 0
        self._calls("dv_pressure_solve_ex", flags, C.byref(it) if self.track_iterations else None)
        if flags:
            self._fused_vis = self._fusion_mark(self._VIS_READS)
        self.last_iters = (self.last_iters[0], it.value)

    track_iterations = False
    compute_vis = False  # KarmanVortexSolver sets it from the scene (computeVis)

    # ----------------------------------------------------------- DIMCV
    def compute_v_star(self):  # :264-271 (computed with vorticity and ∇v)
        self._calls("dv_dimcv_vorticity")

    def compute_vorticity(self):  # :284-293
        self._calls("dv_dimcv_vorticity")

    def compute_grad_v(self):  # :273-282
        self._calls("dv_dimcv_vorticity")

    def init(self):  # :803-806 — one sweep for v*, ω and ∇v, and Δω (:573-583) with them
        self._calls("dv_vorticity_dvort")
        self._fused_dvort = self._fusion_mark(self._DVORT_READS, ("v_star",))

    def compute_d_vorticity(self):  # :573-583
        if self._fusion_fresh(self._fused_dvort, self._DVORT_READS, ("v_star",)):
            return  # computed by init's sweep, bit-identical
        self._calls("dv_d_vorticity")

    def compute_all_d_vort_smoothed(self):  # :666-677
        self._calls("dv_smooth_d_vort")

    def compute_kinematic_vorticity_num_sample(self):  # :305-324
        bd = 1 if self.sampler == "bernoulli" else 0
        self._calls("dv_kvn_sample", self.seed, self.rng_step, bd)

    def record_vort_part_sample_idx(self):  # :326-335
        if self.sampler == "bernoulli":
            self._calls("dv_record_samples")

    def update_sample(self):  # :808-810
        self.compute_kinematic_vorticity_num_sample()
        self.record_vort_part_sample_idx()

    def compute_kernel_density(self):  # :738-751
        self._calls("dv_akde")

    def _draw_samples(self):
        if self.sampler in ("inverse_cdf", "stratified"):
            M = self.mc_samples
            if M is None:
                M = 1.0 / 16.0
            if isinstance(M, float) and M <= 1.0:
                M = max(1, int(M * self.ps.fluid_particle_num[None]))
            self._calls("dv_sample", _MODES[self.sampler], self.seed, self.rng_step, int(M))
        elif self.sampler == "injected":
            self._calls("dv_sample", DV_SAMPLE_INJECTED, 0, 0, int(self.injected_num_samples))

    autotune = True
    far_tile = None

    def vort2vel(self):  # :679-719
        if self.far_tile is None:
            import os
            forced = os.environ.get("DIMCV_FAR_TT")
            if forced:
                self.far_tile = int(forced)
                _lib.check(self.ctx, self.lib.dv_set_far_tile(self.ctx, self.far_tile), "dv_set_far_tile")
            elif self.autotune:
                # one-time choice of the far-field tile (targets per thread) on this state
                tt, ms = C.c_int32(0), C.c_float(0)
                self._calls("dv_autotune", C.byref(tt), C.byref(ms))
                self.far_tile = tt.value or 4
            else:
                self.far_tile = 4
        self._calls("dv_vvpe_mc")

    def update_particle_life_time(self):  # :753-760
        self._call("dv_life_time")

    def copy_x_temp(self):  # :797-801 (with compute_vorticity_vis)
        if self._fusion_fresh(self._fused_vis, self._VIS_READS):
            return  # computed by pressure_solve's opening sweep, bit-identical
        self._calls("dv_vis")

    def compute_vorticity_vis(self):  # :785-795 — done by copy_x_temp's fused sweep
        pass

    def smooth_and_kernel_density(self):
        """compute_all_d_vort_smoothed + compute_kernel_density (:660-677,
        738-751) in one sweep; needs this step's KVN (update_sample first)."""
        self._calls("dv_smooth_akde")

    def dimcv(self):  # :812-819
        self.init()
        self.compute_d_vorticity()
        # KVN and the birth/death draws read only ∇v, life time and the sample
        # flags, and the smoothing reads none of what they write, so they run
        # first and the smoothing shares the AKDE's neighbour sweep
        self.update_sample()
        self.smooth_and_kernel_density()
        self._draw_samples()
        self.vort2vel()
        self.update_particle_life_time()
        self.rng_step += 1

    # ----------------------------------------------------------- emission
    def emit_particle(self):  # :616-637
        for emitter in self.ps.fluid_emitters:
            obj_id = emitter["objectId"]
            center = np.array(emitter["squareCenter"])
            size = np.array(emitter["squareSize"])
            init_v = np.array(emitter["velocity"])
            lower = center - 0.5 * size
            cube = size + self.ps.particle_radius * np.abs(init_v) / np.linalg.norm(init_v)
            self.ps.object_collection[obj_id]["particleNum"] += self.ps.compute_cube_particle_num(lower, lower + cube)
            self.ps.add_cube(object_id=obj_id, lower_corner=lower, cube_size=cube, velocity=init_v,
                             density=emitter["density"], is_dynamic=1, color=emitter["color"], material=1)

    def dump_num_particles_each_emitters_ti2np(self):  # :639-642
        """Emitter bookkeeping is computed on demand (ps.num_particles_each_emitter)
        instead of a device read every step."""

    def dump_num_particles_each_emitters_np2ti(self):  # :644-647
        """See dump_num_particles_each_emitters_ti2np."""
