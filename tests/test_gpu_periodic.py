"""Periodic box (new option): minimum-image neighbours, sweeps, VVPE and
full Biot-Savart on the GPU against the oracle, and the wrap of advection."""
import ctypes as C

import numpy as np
import pytest
import torch

from dimcv_sph_b200 import scenes
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu


def relerr(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


@pytest.fixture(scope="module")
def box(cuda):
    from dimcv_sph_b200.dimcv_sph import DIMCVSPHSolver
    from dimcv_sph_b200.particle_system import ParticleSystem
    cfg, x, w = scenes.periodic2d(4096, seed=2)
    n = x.shape[0]
    ps = ParticleSystem(cfg, capacity=n)
    rng = np.random.default_rng(4)
    v = rng.normal(0, 0.2, size=x.shape).astype(np.float32)
    ps.add_particles(0, n, x, v, np.full(n, 1000.0), np.zeros(n), np.ones(n, np.int32), np.ones(n, np.int32),
                     np.zeros((n, 3), np.int32))
    solver = DIMCVSPHSolver(ps)
    solver.initialize()
    perm = ps.permutation()
    solver.d_vort_smoothed[:n, 2] = torch.from_numpy(w[perm]).to(ps.device)
    return ps, solver


def mirror(ps):
    o = OracleSim(ps.params, ps.particle_max_num, 0)
    o.load_snapshot(ps.snapshot(), ps.counters())
    o.counting_sort()
    assert np.array_equal(o.permutation(), np.arange(o.counters()["n"]))
    return o


def test_periodic_neighbours_and_sweeps_bitexact(box):
    ps, solver = box
    o = mirror(ps)
    off, nbr = (t.cpu().numpy() for t in ps.neighbor_lists())
    ooff, onbr = o.neighbor_lists()
    assert np.array_equal(off, ooff) and np.array_equal(nbr, onbr)
    # wrap-around pairs exist: some neighbours are more than half a box apart in raw x
    x = ps.snapshot()["x"]
    i = np.repeat(np.arange(len(off) - 1), np.diff(off))
    raw = np.abs(x[i] - x[nbr])
    assert np.any(raw > 0.5)
    # every particle of a jittered lattice has neighbours on all sides
    assert np.min(np.diff(off)) >= 6
    for meth, op, field in (("compute_densities", "densities", "density"),
                            ("compute_DFSPH_factor", "dfsph_factor", "dfsph_factor")):
        getattr(solver, meth)()
        o.call(op)
        g, r = ps.snapshot()[field], o.snapshot()[field]
        assert np.array_equal(g, r), field


def test_periodic_vvpe_and_bs(box):
    ps, solver = box
    n = ps.particle_num[None]
    solver.init()
    solver.compute_kinematic_vorticity_num_sample()
    solver.compute_kernel_density()
    solver.mc_samples = n // 8
    solver._draw_samples()
    o = mirror(ps)
    solver.vort2vel()
    o.calls("vvpe_mc", 64)
    g, r = ps.snapshot(), o.snapshot()
    assert np.max(np.abs(r["solver.v_vort"])) > 0
    assert relerr(g["solver.v_vort"][:, :3], r["solver.v_vort"][:, :3]) < 1e-5
    # full BS with minimum image, FP64 on the GPU against the oracle
    om = np.zeros((ps.particle_max_num, 4), np.float32)
    om[:n, 2] = solver.d_vort_smoothed[:n, 2].cpu().numpy()
    om_d = torch.from_numpy(om).to(ps.device)
    out = torch.zeros((n, 4), dtype=torch.float64, device=ps.device)
    rc = ps.lib.dv_bs_full(ps.ctx, C.byref(ps.fields_struct), C.c_void_p(om_d.data_ptr()), None, n,
                           C.c_void_p(out.data_ptr()), 64)
    assert rc == 0
    ref = o.bs_full(om, None, n)
    assert relerr(out.cpu().numpy()[:, :2], ref[:, :2]) < 1e-12


def test_periodic_advect_wraps(box):
    ps, solver = box
    n = ps.particle_num[None]
    ps.v[:n] = torch.tensor([3.0, -7.0], device=ps.device)  # several cells per step at dt = 1e-3... x100
    solver._set_dt(0.05)
    solver.advect()
    x = ps.x[:n].cpu().numpy()
    assert x.min() >= 0.0 and x.max() < 1.0
    ps.initialize_particle_system()
    assert ps.counters()["n"] == n and ps.counters()["status"] & 4 == 0  # nothing outside the grid
