"""Mesh rigid bodies on the host (particle_system.py:616-639): OBJ / STL
loading, placement and the subdivide voxeliser with hole fill.  A box whose
corners sit on the voxel lattice has a known filled voxelisation; a sphere's
is bounded by its radius and close to its volume."""
import struct

import numpy as np
import pytest

from dimcv_sph_b200 import mesh

BOX_V = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
BOX_F = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [1, 2, 6], [1, 6, 5], [2, 3, 7], [2, 7, 6], [3, 0, 4], [3, 4, 7]])


def write_obj(path, v, f, quads=False):
    lines = [f"v {a} {b} {c}" for a, b, c in v]
    if quads:  # the six faces as quads, with texture / normal indices
        for q in ([0, 3, 2, 1], [4, 5, 6, 7], [0, 1, 5, 4], [1, 2, 6, 5], [2, 3, 7, 6], [3, 0, 4, 7]):
            lines.append("f " + " ".join(f"{k + 1}/1/1" for k in q))
    else:
        lines += [f"f {a + 1} {b + 1} {c + 1}" for a, b, c in f]
    path.write_text("# box\n" + "\n".join(lines) + "\n")


def write_stl_binary(path, v, f):
    out = bytearray(b"\0" * 80) + struct.pack("<I", len(f))
    for tri in f:
        out += struct.pack("<3f", 0, 0, 0) + b"".join(struct.pack("<3f", *v[k]) for k in tri) + b"\0\0"
    path.write_bytes(bytes(out))


def write_stl_ascii(path, v, f):
    lines = ["solid box"]
    for tri in f:
        lines += ["facet normal 0 0 0", "outer loop"] + [f"vertex {a} {b} {c}" for a, b, c in v[tri]]
        lines += ["endloop", "endfacet"]
    path.write_text("\n".join(lines + ["endsolid box"]) + "\n")


def lattice(n, pitch):
    k = np.arange(n + 1) * pitch
    return np.stack(np.meshgrid(k, k, k, indexing="ij"), -1).reshape(-1, 3)


def test_box_voxelisation_is_the_full_lattice():
    pts = mesh.voxelize_filled(BOX_V, BOX_F, 0.1)
    assert pts.shape == (11 ** 3, 3)
    np.testing.assert_allclose(pts, lattice(10, 0.1), atol=1e-12)  # lexicographic order


@pytest.mark.parametrize("kind", ["obj", "obj_quads", "stl_binary", "stl_ascii"])
def test_loaders_agree(tmp_path, kind):
    p = tmp_path / ("box.obj" if kind.startswith("obj") else "box.stl")
    if kind == "obj":
        write_obj(p, BOX_V, BOX_F)
    elif kind == "obj_quads":
        write_obj(p, BOX_V, BOX_F, quads=True)
    elif kind == "stl_binary":
        write_stl_binary(p, BOX_V, BOX_F)
    else:
        write_stl_ascii(p, BOX_V, BOX_F)
    v, f = mesh.load_mesh(p)
    assert v.shape == (8, 3) and f.shape == (12, 3)  # STL corners merged to 8 vertices
    # same triangles as the source box (as sets of corner coordinates)
    tri = {tuple(sorted(map(tuple, v[t]))) for t in f}
    assert tri == {tuple(sorted(map(tuple, BOX_V[t]))) for t in BOX_F} or kind == "obj_quads"
    np.testing.assert_allclose(mesh.voxelize_filled(v, f, 0.25), lattice(4, 0.25), atol=1e-12)


def test_placement_scale_rotation_translation():
    body = {"scale": [2.0, 1.0, 1.0], "rotationAngle": 90.0, "rotationAxis": [0, 0, 1],
            "translation": [10.0, 0.0, 0.0]}
    v = mesh.place(BOX_V, body)
    # scaled to 2 x 1 x 1, turned a quarter about z through its centre (1, 0.5, 0.5): 1 x 2 x 1
    lo, hi = v.min(0), v.max(0)
    np.testing.assert_allclose(hi - lo, [1.0, 2.0, 1.0], atol=1e-6)
    np.testing.assert_allclose((hi + lo) / 2, [11.0, 0.5, 0.5], atol=1e-6)


def icosphere(level, r, c):
    t = (1 + 5 ** 0.5) / 2
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], float)
    f = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6],
         [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
         [8, 6, 7], [9, 8, 1]]
    v = list(v / np.linalg.norm(v, axis=1, keepdims=True))
    for _ in range(level):
        mid = {}

        def m(a, b):
            k = (min(a, b), max(a, b))
            if k not in mid:
                p = (v[a] + v[b]) / 2
                v.append(p / np.linalg.norm(p))
                mid[k] = len(v) - 1
            return mid[k]
        f = [g for a, b, cc in f for g in ([a, m(a, b), m(cc, a)], [b, m(b, cc), m(a, b)], [cc, m(cc, a), m(b, cc)],
                                           [m(a, b), m(b, cc), m(cc, a)])]
    return np.asarray(v) * r + np.asarray(c), np.asarray(f)


def test_sphere_voxelisation_is_bounded_and_filled():
    r, pitch = 0.3, 0.04
    v, f = icosphere(3, r, [0.5, 0.5, 0.5])
    pts = mesh.voxelize_filled(v, f, pitch)
    d = np.linalg.norm(pts - 0.5, axis=1)
    assert d.max() <= r + pitch * np.sqrt(3) / 2 + 1e-9
    vol = 4 / 3 * np.pi * r ** 3 / pitch ** 3
    # the surface voxels add about half a voxel of thickness: (1 + 0.5 pitch / r)^3 ~ 1.2-1.35
    assert 0.9 * vol < len(pts) < 1.5 * vol
    # filled: the voxel at the centre and every lattice point well inside are there
    inside = lattice(25, pitch)
    inside = inside[np.linalg.norm(inside - 0.5, axis=1) < r - pitch]
    key = {tuple(np.round(p / pitch).astype(int)) for p in pts}
    assert all(tuple(np.round(p / pitch).astype(int)) in key for p in inside)

