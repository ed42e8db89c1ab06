"""bounceBackBoundary (sph_base.py:118-179, karman_vortex.py:226-230):
enforce_boundary on the GPU against the oracle (positions and velocities
bit-exact, 2-D and 3-D, particles beyond every face, on a face, in a corner,
solids and non-dynamic fluid untouched), and the option in a channel run."""
import ctypes as C

import numpy as np
import pytest

from dimcv_sph_b200 import scenes
from dimcv_sph_b200.config_builder import SimConfig
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu


def box_cfg(dim):
    c = {"domainStart": [0.0] * dim, "domainEnd": [1.0] * dim, "particleRadius": 0.02, "density0": 1000,
         "timeStepSize": 1e-3, "gravitation": [0.0] * dim, "reservedCapacity": 400}
    return SimConfig(config={"Configuration": c})


@pytest.mark.parametrize("dim", [2, 3])
def test_enforce_boundary_matches_oracle(cuda, dim):
    from dimcv_sph_b200.dimcv_sph import DIMCVSPHSolver
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(box_cfg(dim))
    rng = np.random.default_rng(7)
    n = 300
    x = rng.uniform(-0.1, 1.1, size=(n, dim)).astype(np.float32)
    x[0] = 0.08   # exactly on the lower bound (padding = h = 0.08): clamped, counted as a hit
    x[1] = 1.5    # beyond every upper face: a corner
    v = rng.normal(0, 1, size=(n, dim)).astype(np.float32)
    mat = np.where(rng.uniform(size=n) < 0.8, 1, 0).astype(np.int32)
    dyn = np.where(rng.uniform(size=n) < 0.9, 1, 0).astype(np.int32)
    dyn[mat == 0] = 0
    ps.add_particles(0, n, x, v, np.full(n, 1000.0), np.zeros(n), mat, dyn, np.zeros((n, 3), np.int32))
    solver = DIMCVSPHSolver(ps)
    o = OracleSim(ps.params, ps.particle_max_num, 0)
    o.load_snapshot(ps.snapshot(), ps.counters())
    before = ps.snapshot()
    solver.enforce_boundary_3D(1)
    pad = np.float32(ps.padding)
    lo = (C.c_float * 3)(*([float(pad)] * 3))
    hi = (C.c_float * 3)(*[float(np.float32(np.float32(ps.domain_size[d]) - pad)) if d < dim else 0.0
                           for d in range(3)])
    assert o.lib.dvo_enforce_boundary(o.ctx, o._fp(), 1, lo, hi) == 0
    g, r = ps.snapshot(), o.snapshot()
    for k in ("x", "v"):
        assert np.array_equal(g[k][:n].view(np.int32), r[k][:n].view(np.int32)), k
    moved = np.any(g["x"][:n] != before["x"][:n], axis=1)
    assert moved.sum() > 20 and np.all((g["material"][:n][moved] == 1) & (g["is_dynamic"][:n][moved] == 1))
    fl = (g["material"][:n] == 1) & (g["is_dynamic"][:n] == 1)
    xf = g["x"][:n][fl][:, :dim]
    assert np.all(xf >= pad) and np.all(xf <= np.float32(1.0) - pad)


def test_channel_with_bounce_back(cuda):
    from dimcv_sph_b200.particle_system import ParticleSystem
    cfg = scenes.channel2d(trim_cylinder=True)
    cfg.config["Configuration"]["bounceBackBoundary"] = True
    ps = ParticleSystem(cfg)
    solver = ps.build_solver()
    solver.initialize()
    for _ in range(3):
        solver.step()
    s = ps.snapshot()
    fl = (s["material"] == 1) & (s["is_dynamic"] == 1) & (s["is_active"] == 1)
    pad = np.float32(ps.padding)
    assert fl.sum() > 1000
    xf = s["x"][fl][:, :2]
    assert np.all(xf >= pad) and np.all(xf[:, 0] <= np.float32(4.0) - pad)
