"""A static mesh rigid body (particle_system.py:90-97, 276-303, 616-639) in a
3-D box: its voxel particles become static boundary particles of the scene,
and the boundary volume, densities and DFSPH factor of the scene are
bit-exact with the oracle on the same particles."""
import numpy as np
import pytest

from dimcv_sph_b200 import mesh
from dimcv_sph_b200.config_builder import SimConfig
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu

BOX_V = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
BOX_F = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [1, 2, 6], [1, 6, 5], [2, 3, 7], [2, 7, 6], [3, 0, 4], [3, 4, 7]])


def test_static_mesh_rigid_body(cuda, tmp_path):
    from dimcv_sph_b200.dimcv_sph import DIMCVSPHSolver
    from dimcv_sph_b200.particle_system import ParticleSystem
    obj = tmp_path / "block.obj"
    obj.write_text("\n".join([f"v {a} {b} {c}" for a, b, c in BOX_V] +
                             [f"f {a + 1} {b + 1} {c + 1}" for a, b, c in BOX_F]) + "\n")
    body = {"objectId": 5, "geometryFile": str(obj), "scale": [0.2, 0.2, 0.2], "translation": [0.4, 0.4, 0.1],
            "rotationAngle": 30.0, "rotationAxis": [0.0, 0.0, 1.0], "isDynamic": False, "density": 1000.0,
            "color": [50, 50, 50], "velocity": [0.0, 0.0, 0.0]}
    cfg = SimConfig(config={
        "Configuration": {"domainStart": [0.0, 0.0, 0.0], "domainEnd": [1.0, 1.0, 1.0], "particleRadius": 0.02,
                          "density0": 1000, "timeStepSize": 1e-3, "gravitation": [0.0, 0.0, -9.81],
                          "volumeScale": 1.0, "samplerMode": "inverse_cdf", "mcSamples": 1.0 / 16.0},
        "FluidBlocks": [{"objectId": 0, "start": [0.1, 0.1, 0.35], "end": [0.9, 0.9, 0.6],
                         "translation": [0.0, 0.0, 0.0], "scale": [1.0, 1.0, 1.0], "velocity": [0.0, 0.0, 0.0],
                         "density": 1000.0, "color": [0, 0, 255]}],
        "RigidBodies": [body]})
    expect = mesh.rigid_body_points(dict(body), 0.04)
    ps = ParticleSystem(cfg)
    solver = DIMCVSPHSolver(ps)
    solver.initialize()  # static boundary volume (sph_base.py:91-98)
    ps.initialize_particle_system()
    c = ps.counters()
    assert c["n_solid"] == len(expect) > 100
    snap = ps.snapshot()
    solid = snap["material"] == 0
    got = snap["x"][solid][:, :3]
    key = lambda a: set(map(tuple, np.round(np.asarray(a, np.float64) / 1e-6).astype(np.int64)))
    assert key(got) == key(expect.astype(np.float32))
    assert np.all(snap["object_id"][solid] == 5)
    o = OracleSim(ps.params, ps.particle_max_num, 0)
    o.load_snapshot(ps.snapshot(), ps.counters())
    o.counting_sort()
    assert np.array_equal(o.permutation(), np.arange(o.counters()["n"]))
    for meth, op, field in (("compute_densities", "densities", "density"),
                            ("compute_DFSPH_factor", "dfsph_factor", "dfsph_factor")):
        getattr(solver, meth)()
        o.call(op)
        assert np.array_equal(ps.snapshot()[field], o.snapshot()[field]), field
    # the solids' volumes come from the boundary-volume pass of the same run
    assert np.all(np.isfinite(snap["m_V"][solid])) and np.all(snap["m_V"][solid] > 0)
