"""The 3-D per-step neighbour lists as the grid build stores them (the lists
every sweep reads) against the oracle's for_all_neighbors order
(particle_system.py:562-586): the sphere scene, a dense particle block and a
clump whose particles have more neighbours than the 64 fixed slots of the
build's first pass, and a solid outside the grid whose window is not its
(clamped) key cell.  Bit-exact offsets and entries."""
import numpy as np
import pytest

from dimcv_sph_b200 import scenes
from dimcv_sph_b200.config_builder import SimConfig
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu


def oracle_lists(ps):
    o = OracleSim(ps.params, ps.particle_max_num, 0)
    o.load_snapshot(ps.snapshot(), ps.counters())
    o.counting_sort()
    assert np.array_equal(o.permutation(), np.arange(o.counters()["n"]))
    return o.neighbor_lists()


def check_stored(ps):
    """Every row the step walks (fluid and dynamic solids) equals the
    oracle's; the rows of static solids are stored empty.  The cell-scan
    export has every row and equals the oracle."""
    off, nbr = (t.cpu().numpy() for t in ps.stored_neighbor_lists())
    ooff, onbr = oracle_lists(ps)
    n = ooff.size - 1
    snap = ps.snapshot()
    static = (snap["material"][:n] == 0) & (snap["is_dynamic"][:n] == 0)
    cnt, ocnt = np.diff(off), np.diff(ooff)
    assert np.all(cnt[static] == 0), "static solid rows"
    assert np.array_equal(cnt[~static], ocnt[~static]), "row lengths"
    keep = np.repeat(~static, ocnt)
    assert np.array_equal(nbr, onbr[keep]), "entries"
    eoff, enbr = (t.cpu().numpy() for t in ps.neighbor_lists())
    assert np.array_equal(eoff, ooff) and np.array_equal(enbr, onbr)
    return ooff, static


def test_sphere_scene_lists(cuda):
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(scenes.sphere3d(radius=0.016, dt=6.4e-4))
    ps.initialize_particle_system()
    off, static = check_stored(ps)
    c = np.diff(off)
    assert ps.counters()["n"] > 40000 and c.max() <= 64 and c.mean() > 20
    assert static.sum() > 1000  # the sphere and the walls


def box3d(reserved):
    c = {"domainStart": [0.0, 0.0, 0.0], "domainEnd": [1.0, 1.0, 1.0], "particleRadius": 0.02, "density0": 1000,
         "timeStepSize": 1e-3, "gravitation": [0.0, 0.0, 0.0], "volumeScale": 1.0, "reservedCapacity": reserved,
         "samplerMode": "inverse_cdf", "mcSamples": 1.0 / 16.0}
    return SimConfig(config={"Configuration": c})


def add(ps, x, material):
    x = np.asarray(x, np.float32)
    n = x.shape[0]
    ps.add_particles(0, n, x, np.zeros_like(x), np.full(n, 1000.0), np.zeros(n), np.full(n, material, np.int32),
                     np.ones(n, np.int32), np.zeros((n, 3), np.int32))


def test_dense_block_crowded_particle_and_clamped_solid(cuda):
    """h = 0.08 = one cell: 4000 particles in a 0.3-wide cube have about 300
    neighbours each (more than the 64 fixed slots), as do the particles of
    the 80-particle clump; the solid at x = 1.3 sits outside the grid
    (clamped key cell, window from its position)."""
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(box3d(reserved=40000))  # room for ~1.3M list entries (48 per slot)
    rng = np.random.default_rng(11)
    spread = rng.uniform(0.05, 0.95, size=(800, 3))
    dense = rng.uniform(0.35, 0.65, size=(4000, 3))
    clump = 0.15 + rng.uniform(-0.01, 0.01, size=(80, 3))
    add(ps, np.concatenate([spread, dense, clump]), 1)
    add(ps, [[1.3, 0.5, 0.5], [0.97, 0.5, 0.5]], 0)
    ps.initialize_particle_system()
    assert ps.counters()["status"] & 4  # a particle outside the grid
    off, _ = check_stored(ps)
    assert np.diff(off).max() > 64
