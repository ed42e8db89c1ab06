"""Dynamic rigid particles (isDynamic rigid blocks): the moving boundary
volume (sph_base.py:105-112), gravity and the pressure solve's reaction
(dimcv_sph.py:540-549) drive them through advect (:210-218).  Three steps of
a fluid box with a dynamic block in it, compared with the oracle after every
stage: the reaction is gathered per solid in the same order on both, so the
fields are bit-exact."""
import numpy as np
import pytest

from dimcv_sph_b200.config_builder import SimConfig
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu


def block(oid, start, end, dynamic, density=1000.0):
    return {"objectId": oid, "start": start, "end": end, "translation": [0.0, 0.0, 0.0], "scale": [1.0, 1.0, 1.0],
            "velocity": [0.0, 0.0, 0.0], "density": density, "color": [0, 0, 0], "isDynamic": dynamic}


def bits(a):
    return np.ascontiguousarray(a).view(np.int32)


def test_dynamic_rigid_block_steps_match_oracle(cuda):
    from dimcv_sph_b200.dimcv_sph import DIMCVSPHSolver
    from dimcv_sph_b200.particle_system import ParticleSystem
    cfg = SimConfig(config={
        "Configuration": {"domainStart": [0.0, 0.0, 0.0], "domainEnd": [1.0, 1.0, 1.0], "particleRadius": 0.02,
                          "density0": 1000, "timeStepSize": 1e-3, "gravitation": [0.0, 0.0, -9.81],
                          "volumeScale": 1.0},
        "FluidBlocks": [block(0, [0.1, 0.1, 0.1], [0.9, 0.9, 0.45], False)],
        "RigidBlocks": [block(1, [0.0, 0.0, 0.0], [1.0, 1.0, 0.08], False),
                        block(3, [0.4, 0.4, 0.46], [0.6, 0.6, 0.56], True, density=500.0)]})
    ps = ParticleSystem(cfg)
    assert ps.has_dynamic_rigid
    solver = DIMCVSPHSolver(ps)
    solver.initialize()
    moved = 0.0
    for step in range(3):
        ps.initialize_particle_system()
        o = OracleSim(ps.params, ps.particle_max_num, 0)
        o.lib.dvo_set_dynamic_rigid(o.ctx, 1)
        o.load_snapshot(ps.snapshot(), ps.counters())
        o.counting_sort()
        assert np.array_equal(o.permutation(), np.arange(o.counters()["n"]))
        x0 = ps.snapshot()["x"]
        stages = [("compute_moving_boundary_volume", lambda: o.call("moving_boundary_volume"), ["m_V"]),
                  ("compute_densities", lambda: o.call("densities"), ["density"]),
                  ("compute_DFSPH_factor", lambda: o.call("dfsph_factor"), ["dfsph_factor"]),
                  ("divergence_solve", o.divergence_solve, ["v", "density_adv"]),
                  ("compute_non_pressure_forces", lambda: o.call("nonpressure"), ["acceleration"]),
                  ("predict_velocity", lambda: o.call("predict_velocity"), ["v"]),
                  ("pressure_solve", o.pressure_solve, ["v", "acceleration", "density_adv"]),
                  ("advect", lambda: o.call("advect"), ["x", "v"])]
        for meth, ocall, fields in stages:
            getattr(solver, meth)()
            ocall()
            g, r = ps.snapshot(), o.snapshot()
            for k in fields:
                assert np.array_equal(bits(g[k]), bits(r[k])), (step, meth, k)
        s = ps.snapshot()
        dyn = (s["material"] == 0) & (s["is_dynamic"] == 1)
        assert dyn.sum() > 50
        moved = max(moved, float(np.abs(s["x"][dyn] - x0[dyn]).max()))
    assert moved > 0  # the dynamic block moves; the static floor does not
    s = ps.snapshot()
    floor = (s["material"] == 0) & (s["is_dynamic"] == 0)
    assert np.all(s["acceleration"][floor] == 0)
