"""Host-side parameter derivation and scene builders (no GPU)."""
import numpy as np
import pytest

from dimcv_sph_b200 import scenes
from dimcv_sph_b200.params import f32_pow_int, make_params, sqrt_limits


@pytest.mark.parametrize("h", [0.04, 0.016, 0.018, 0.0390625, 1e-3, 3.3e-2])
def test_sqrt_limits_are_exact(h):
    lo, hi = sqrt_limits(h)
    h32 = np.float32(h)
    lo32, hi32 = np.float32(lo), np.float32(hi)
    assert np.sqrt(lo32) >= h32 and np.sqrt(np.nextafter(lo32, np.float32(0))) < h32
    assert np.sqrt(hi32) <= h32 and np.sqrt(np.nextafter(hi32, np.float32(np.inf))) > h32
    # exhaustive check on the f32 values around h^2
    t = np.float32(h32 * h32)
    for k in range(-64, 65):
        v = t
        step = np.float32(np.inf) if k > 0 else np.float32(0)
        for _ in range(abs(k)):
            v = np.nextafter(v, step)
        assert (np.sqrt(v) < h32) == (v < lo32)
        assert (np.sqrt(v) > h32) == (v > hi32)


def test_pow_by_squaring():
    h = np.float32(25.0)
    assert f32_pow_int(h, 2) == np.float32(h * h)
    assert f32_pow_int(h, 3) == np.float32(np.float32(h * h) * h)


def test_channel_params_follow_reference_expressions():
    cfg = scenes.channel2d()
    p = make_params(cfg)
    assert p.dim == 2 and list(p.grid_num)[:2] == [100, 25]
    assert p.support_radius == np.float32(0.04)
    assert p.kW == np.float32(np.float32(1.8189) * np.float32(np.float32(25.0) * np.float32(25.0)))
    assert p.kW2 == np.float32(2) * np.float32(p.kW)
    assert p.neighbor_min == 7
    dt = float(np.float32(4e-4))
    assert p.inv_dt == np.float32(1.0 / dt)
    assert abs(p.eta_div - (1.0 / dt) * 0.1 * 0.01 * 1000) < 1e-9
    assert p.eta_p == 0.05 * 0.01 * 1000
    assert p.visc_coef == np.float32(np.float32(8) * np.float32(1e-3))
    assert p.has_transit == 1 and p.transit_span == np.float32(0.02)
    assert p.skip_cell0 == 1 and p.kernel_mode == 0


def test_sphere_grid_matches_config():
    cfg = scenes.sphere3d()
    p = make_params(cfg)
    assert list(p.grid_num) == [188, 63, 63]
    assert p.neighbor_min == 20


def test_ring_scene_volume_and_offset():
    cfg, x, w = scenes.ring3d(4096, seed=1)
    p = make_params(cfg)
    assert p.cell_origin_offset == 1 and p.skip_cell0 == 0 and p.kernel_mode == 1
    assert x.shape == (4096, 3) and np.all(np.abs(x) <= 1.0)
    r = 0.5 * (8.0 / 4096) ** (1 / 3)
    vp = 1.25 * 0.8 * (2 * r) ** 3
    assert abs(vp - 8.0 / 4096) < 1e-12
    # the ring peak vorticity is Γ/(πσ²) on the core circle
    c = np.array([[0.5, 0.0, 0.0]])
    assert abs(np.linalg.norm(scenes.ring_vorticity(c)) - 1.0 / (np.pi * 0.05 ** 2)) < 1e-9


def test_periodic_box_grid():
    cfg, x, w = scenes.periodic2d(65536, seed=0)
    p = make_params(cfg)
    # h = 4 r = 2/256; cells of 1/floor(1/h) = 1/128 >= h
    assert p.periodic == 1 and p.cell_origin_offset == 1 and p.skip_cell0 == 0
    assert list(p.grid_num)[:2] == [128, 128]
    assert p.grid_size == np.float32(1.0 / 128) and p.grid_size >= p.support_radius
    assert list(p.box)[:2] == [1.0, 1.0]
    assert x.shape == (65536, 2) and x.min() >= 0.0 and x.max() < 1.0
    vp = 1.25 * 0.8 * (2 * (0.5 / 256)) ** 2
    assert abs(vp - 1.0 / 65536) < 1e-15
    # the blobs are periodic: the field at x and x + (1, 0) agree
    a = scenes.periodic_blobs(np.array([[0.01, 0.3]]), 1)
    b = scenes.periodic_blobs(np.array([[1.01, 0.3]]), 1)
    assert abs(a[0] - b[0]) < 1e-12


def test_periodic_box_rejects_bad_shapes():
    from dimcv_sph_b200.config_builder import SimConfig
    base = {"domainStart": [0.0, 0.0], "domainEnd": [1.0, 0.5], "particleRadius": 0.03,
            "density0": 1000, "timeStepSize": 1e-3, "gravitation": [0, 0], "periodic": True}
    # 1/0.12 -> 8 cells of 0.125, 0.5/0.12 -> 4 cells: too few and not the same size
    with pytest.raises(ValueError):
        make_params(SimConfig(config={"Configuration": base}))


def test_channel_batch_configs():
    import math
    from dimcv_sph_b200.batch import channel_batch_configs, _grid_of
    cfgs, Ns = channel_batch_configs(n_scenes=64, seed=1)
    assert len(cfgs) == 64 and Ns.min() >= 2000 and Ns.max() <= 60000
    # log-uniform: the median of log N sits near the middle of [log 2k, log 60k]
    mid = 0.5 * (math.log(2000) + math.log(60000))
    assert abs(float(np.median(np.log(Ns))) - mid) < 0.5
    grids = np.stack([_grid_of(c) for c in cfgs])
    for c in cfgs:
        g = c.get_cfg
        L, H = g("domainEnd")
        assert abs(L - 4 * H) < 1e-9
        u = c.get_fluid_emitters()[0]["velocity"][0]
        assert 0.5 <= u <= 2.0
        r = g("cylinderRadius")  # U(0.05, 0.15), capped at a quarter of the height
        assert r <= 0.15 + 1e-12 and r <= 0.25 * H + 1e-12
        assert r >= min(0.05, 0.25 * H) - 1e-12
        assert g("particleRadius") == 0.01 and g("timeStepSize") == 4e-4
        assert g("computeVis") is False and g("samplerMode") == "inverse_cdf"
    # the shared batch grid is the largest scene grid
    assert np.all(grids.max(axis=0) >= grids)


def test_scene_without_a_domain_is_a_clear_error():
    """A scene of the reference's vortex-segment solver (SegmentConfiguration,
    no Configuration.domainStart) is refused with a message, not a TypeError."""
    import pytest
    from dimcv_sph_b200.config_builder import SimConfig
    cfg = SimConfig(config={"Configuration": {"particleRadius": 0.01, "timeStep": 0.002},
                            "SegmentConfiguration": {"initType": "v_bundle_pair"}})
    with pytest.raises(ValueError, match="segment"):
        make_params(cfg)
