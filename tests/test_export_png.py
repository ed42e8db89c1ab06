"""PNG frames (karman_vortex.py:38-121) drawn without matplotlib: the colour
map, the 2-D and 3-D views and the file written."""
import numpy as np

from dimcv_sph_b200.export import coolwarm, render_frame


def test_coolwarm_ends_and_middle():
    c = coolwarm(np.array([-40.0, -100.0, 0.0, 40.0, 1e9]))
    assert c[0].tolist() == [59, 76, 192] and c[1].tolist() == [59, 76, 192]
    assert c[2].tolist() == [221, 221, 221]
    assert c[3].tolist() == [180, 4, 38] and c[4].tolist() == [180, 4, 38]


def test_2d_frame_places_and_colours_particles(tmp_path):
    x = np.array([[0.0, 0.0], [4.0, 1.0], [2.0, 0.5], [1.0, 0.25]])
    vort = np.array([40.0, -40.0, 0.0, 5.0])
    fluid = np.array([True, True, False, False])
    solid = np.array([False, False, True, False])  # the last is neither: not drawn
    img = render_frame(x, vort, fluid, solid, width=400)
    assert img.size == (400, 100) and img.mode == "RGBA"
    a = np.asarray(img)
    assert a[99, 0].tolist() == [180, 4, 38, 153]      # (0, 0): bottom left, red, alpha 0.6
    assert a[0, 399].tolist() == [59, 76, 192, 153]    # (4, 1): top right, blue
    assert a[50, 200].tolist() == [0, 200, 83, 255]    # the solid, #00C853
    assert (a[..., 3] > 0).sum() == 3
    p = tmp_path / "f.png"
    img.save(p)
    assert p.read_bytes()[:8] == b"\x89PNG\r\n\x1a\n"


def test_3d_frame_draws_the_nearest_particle():
    rng = np.random.default_rng(0)
    x = rng.uniform([0, 0, 0], [4, 1, 1], size=(5000, 3))
    fluid = np.ones(5000, bool)
    img = render_frame(x, rng.normal(0, 20, 5000), fluid, ~fluid, width=800)
    a = np.asarray(img)
    assert img.size == (800, 320) and (a[..., 3] > 0).sum() > 1000
    # two particles on the same ray: the one nearer the viewer wins
    el, az = np.radians(30.0), np.radians(-60.0)
    f = np.array([np.cos(el) * np.cos(az), np.cos(el) * np.sin(az), np.sin(el)])
    c = np.array([2.0, 0.5, 0.5])
    y = np.stack([c + 0.3 * f, c - 0.3 * f])
    b = np.asarray(render_frame(y, np.array([40.0, -40.0]), np.ones(2, bool), np.zeros(2, bool), width=800))
    drawn = b[b[..., 3] > 0]
    assert len(drawn) == 1 and drawn[0].tolist() == [180, 4, 38, 153]
