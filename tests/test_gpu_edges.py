"""Edge cases of the CUDA path: empty and one-particle scenes through the
whole substep, the emission capacity clamp, particles leaving the box or the
grid, an out-of-range injected sample index, a non-finite velocity in a
solve, and out-of-range sizes.  Each is handled by the library's own checks
(a status bit, an error, or the reference's clamp); none reaches memory out
of bounds."""
import ctypes as C

import numpy as np
import pytest
import torch

from dimcv_sph_b200._abi import (DV_SAMPLE_INJECTED, DV_WARN_BAD_INDEX, DV_WARN_CAPACITY, DV_WARN_NAN,
                                 DV_WARN_OUTSIDE_GRID, DvParams)
from dimcv_sph_b200.config_builder import SimConfig

pytestmark = pytest.mark.gpu


def box_cfg(dim=2, reserved=64, **extra):
    lo = [0.0] * dim
    hi = [1.0] * dim
    c = {"domainStart": lo, "domainEnd": hi, "particleRadius": 0.02, "density0": 1000,
         "timeStepSize": 1e-3, "gravitation": [0.0] * dim, "volumeScale": 1.0,
         "reservedCapacity": reserved, "samplerMode": "inverse_cdf", "mcSamples": 1.0 / 16.0}
    c.update(extra)
    return SimConfig(config={"Configuration": c})


def add(ps, x, v=None, material=1):
    x = np.asarray(x, np.float32)
    n = x.shape[0]
    v = np.zeros_like(x) if v is None else np.asarray(v, np.float32)
    ps.add_particles(0, n, x, v, np.full(n, 1000.0), np.zeros(n), np.full(n, material, np.int32),
                     np.ones(n, np.int32), np.zeros((n, 3), np.int32))


def full_substep(solver):
    solver.compute_densities()
    solver.compute_DFSPH_factor()
    solver.divergence_solve()
    solver.compute_non_pressure_forces()
    solver.dimcv()
    solver.predict_velocity()
    solver.pressure_solve()
    solver.advect()


@pytest.mark.parametrize("dim", [2, 3])
def test_empty_scene_runs_every_stage(cuda, dim):
    from dimcv_sph_b200.dimcv_sph import DIMCVSPHSolver
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(box_cfg(dim))
    solver = DIMCVSPHSolver(ps)
    solver.initialize()
    for _ in range(2):
        ps.initialize_particle_system()
        full_substep(solver)
    c = ps.counters()
    assert c["n"] == 0 and c["num_samples"] == 0 and c["status"] & ~0b11 == 0


def test_single_particle(cuda):
    from dimcv_sph_b200.dimcv_sph import DIMCVSPHSolver
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(box_cfg(2))
    add(ps, [[0.5, 0.5]], [[0.3, -0.1]])
    solver = DIMCVSPHSolver(ps)
    solver.initialize()
    ps.initialize_particle_system()
    full_substep(solver)
    c = ps.counters()
    assert c["n"] == 1 and c["n_fluid"] == 1
    rho = np.float32(ps.density[0].item())
    m_V = np.float32(ps.m_V[0].item())
    # no neighbours: ρ = (m_V W(0)) ρ0, W(0) = kW (dimcv_sph.py:126-148)
    assert rho == np.float32(np.float32(m_V * np.float32(ps.params.kW)) * np.float32(1000.0))
    assert np.all(np.isfinite(ps.v[:1].cpu().numpy())) and np.all(np.isfinite(ps.x[:1].cpu().numpy()))


def test_emission_clamps_at_capacity(cuda):
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(box_cfg(2, reserved=10))
    cap = ps.particle_max_num
    add(ps, np.random.default_rng(0).uniform(0.1, 0.9, size=(cap + 7, 2)))
    c = ps.counters()
    assert c["n"] == cap and c["status"] & DV_WARN_CAPACITY
    assert ps.lib.dv_clear_status(ps.ctx) == 0
    assert ps.counters()["status"] == 0


def test_fluid_leaving_the_box_is_dropped_and_solids_outside_the_grid_are_clamped(cuda):
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(box_cfg(2, reserved=32, cellOriginOffset=True, skipCell0=False))
    add(ps, [[0.5, 0.5], [0.52, 0.5], [1.5, 0.5], [0.5, -0.3]])   # two fluid outside the box
    add(ps, [[2.5, 0.5]], material=0)                               # a solid beyond the grid
    ps.initialize_particle_system()
    c = ps.counters()
    assert c["n"] == 3 and c["n_fluid"] == 2 and c["n_solid"] == 1
    assert c["status"] & DV_WARN_OUTSIDE_GRID
    x = ps.x[:3].cpu().numpy()
    assert np.all(np.isfinite(x))


def test_out_of_range_injected_sample_is_ignored(cuda):
    from dimcv_sph_b200.dimcv_sph import DIMCVSPHSolver
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(box_cfg(2, reserved=512))
    rng = np.random.default_rng(1)
    add(ps, rng.uniform(0.05, 0.95, size=(400, 2)), rng.normal(0, 0.3, size=(400, 2)))
    solver = DIMCVSPHSolver(ps)
    solver.initialize()
    ps.initialize_particle_system()
    solver.compute_densities()
    solver.compute_non_pressure_forces()
    solver.init()
    solver.compute_d_vorticity()
    solver.compute_all_d_vort_smoothed()
    solver.compute_kinematic_vorticity_num_sample()
    solver.compute_kernel_density()
    idx = np.array([3, 17, 10**6, 42, -5], np.int32)
    solver.sample_idx[:5] = torch.from_numpy(idx).to(ps.device)
    solver.sampler = "injected"
    solver.injected_num_samples = 5
    solver._calls("dv_sample", DV_SAMPLE_INJECTED, 0, 0, 5)
    solver.far_tile = 4
    solver.vort2vel()
    c = ps.counters()
    assert c["status"] & DV_WARN_BAD_INDEX
    assert np.all(np.isfinite(solver.v_vort[:c["n"]].cpu().numpy()))


def test_non_finite_velocity_stays_local_and_the_solve_ends(cuda):
    """The divergence error passes through max(adv, 0) (dimcv_sph.py:337-374),
    which drops a NaN as Taichi's max does, so one NaN velocity neither stops
    the solve nor spreads: the other particles keep finite velocities and the
    solve ends within max_iter with a finite error."""
    from dimcv_sph_b200.dimcv_sph import DIMCVSPHSolver
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(box_cfg(2, reserved=512))
    rng = np.random.default_rng(2)
    add(ps, rng.uniform(0.05, 0.95, size=(300, 2)), rng.normal(0, 0.5, size=(300, 2)))
    solver = DIMCVSPHSolver(ps)
    solver.initialize()
    ps.initialize_particle_system()
    ps.v[7, 0] = float("nan")
    solver.compute_densities()
    solver.compute_DFSPH_factor()
    solver.divergence_solve()
    c = ps.counters()
    assert 1 <= c["iters_div"] <= ps.params.max_iter_div
    assert np.isfinite(c["err_div"]) and not c["status"] & DV_WARN_NAN
    bad = np.nonzero(~np.isfinite(ps.v[: c["n"]].cpu().numpy()).all(axis=1))[0]
    assert bad.tolist() == [7]


def test_sizes_out_of_range_are_errors(cuda):
    from dimcv_sph_b200 import _lib
    lib = _lib.load()
    p = DvParams()
    p.dim = 2
    p.grid_num[0], p.grid_num[1], p.grid_num[2] = 1 << 14, 1 << 14, 1  # 28 Morton bits
    p.grid_size = 0.04
    assert not lib.dv_create(C.byref(p), 100, None)
    assert b"Morton" in lib.dv_last_error(None)
    p.grid_num[0], p.grid_num[1] = 10, 10
    assert not lib.dv_create(C.byref(p), (1 << 30) + 1, None)
    assert b"capacity" in lib.dv_last_error(None)


def test_particle_with_more_neighbours_than_list_slots(cuda):
    """A crowded 3-D particle (more neighbours than the 64 fixed slots of the
    list build's first pass) gets its CSR list from a second cell scan; the
    sweeps stay bit-exact with the oracle."""
    from dimcv_sph_b200.dimcv_sph import DIMCVSPHSolver
    from dimcv_sph_b200.particle_system import ParticleSystem
    from oracle.oracle import OracleSim
    ps = ParticleSystem(box_cfg(3, reserved=1024))
    rng = np.random.default_rng(5)
    spread = rng.uniform(0.05, 0.95, size=(600, 3))
    cluster = 0.5 + rng.uniform(-0.01, 0.01, size=(80, 3))  # all within h = 0.08 of each other
    add(ps, np.concatenate([spread, cluster]), rng.normal(0, 0.2, size=(680, 3)))
    solver = DIMCVSPHSolver(ps)
    solver.initialize()
    ps.initialize_particle_system()
    o = OracleSim(ps.params, ps.particle_max_num, 0)
    o.load_snapshot(ps.snapshot(), ps.counters())
    o.counting_sort()
    assert np.array_equal(o.permutation(), np.arange(o.counters()["n"]))
    off, _ = o.neighbor_lists()
    assert np.diff(off).max() > 64
    for meth, op, field in (("compute_densities", "densities", "density"),
                            ("compute_DFSPH_factor", "dfsph_factor", "dfsph_factor")):
        getattr(solver, meth)()
        o.call(op)
        assert np.array_equal(ps.snapshot()[field], o.snapshot()[field]), field
    solver.compute_non_pressure_forces()
    o.call("nonpressure")
    assert np.array_equal(ps.snapshot()["acceleration"], o.snapshot()["acceleration"])


def test_unknown_solve_flags_are_errors(cuda):
    """dv_divergence_solve_ex and dv_pressure_solve_ex refuse flags they do not
    know, and DV_SOLVE_VIS without the solver fields, before launching anything."""
    from dimcv_sph_b200._abi import DV_EINVAL, DV_SOLVE_NONPRESSURE, DV_SOLVE_VIS
    from dimcv_sph_b200.dimcv_sph import DIMCVSPHSolver
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(box_cfg(2, reserved=64))
    solver = DIMCVSPHSolver(ps)
    lib, ctx, f = ps.lib, ps.ctx, C.byref(ps.fields_struct)
    launches = solver._launches()
    assert lib.dv_divergence_solve_ex(ctx, f, 8, None) == DV_EINVAL
    assert b"flags" in lib.dv_last_error(ctx)
    assert lib.dv_divergence_solve_ex(ctx, f, DV_SOLVE_VIS, None) == DV_EINVAL
    assert lib.dv_pressure_solve_ex(ctx, f, C.byref(ps.solver_buf.struct), DV_SOLVE_NONPRESSURE, None) == DV_EINVAL
    assert lib.dv_pressure_solve_ex(ctx, f, None, DV_SOLVE_VIS, None) == DV_EINVAL
    assert b"x_temp" in lib.dv_last_error(ctx)
    assert solver._launches() == launches
