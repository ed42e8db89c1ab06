"""Mesh rigid bodies (particle_system.py:616-639) without trimesh.

The reference loads a triangle mesh with trimesh, places it and turns it into
boundary particles with ``mesh.voxelized(pitch).fill().points`` at pitch =
particle diameter.  This module does the same on the host with NumPy/SciPy:

* loading: Wavefront OBJ (``v`` / ``f`` records, polygons fanned into
  triangles) and STL (binary or ASCII); exact duplicate vertices are merged,
  first occurrence first, as trimesh's default processing does;
* placement (particle_system.py:618-628): scale, then a rotation of
  ``rotationAngle`` degrees (converted with the reference's 3.1415926) about
  ``rotationAxis`` through the vertex mean, then the translation;
* voxelisation, restating trimesh's published subdivide method
  (``voxelize_subdivide``: subdivide_to_size with max_edge = pitch / 2 and at
  most 10 rounds, voxel = round(vertex / pitch)), then the ``holes`` fill
  (``scipy.ndimage.binary_fill_holes`` over the occupied box) and the voxel
  centres ``index * pitch``, in lexicographic index order.

trimesh is not installed here, so these points are not pinned against
trimesh's own output; the tests check the construction on meshes whose
voxelisation is known exactly (a box on the voxel lattice) or bounded (a
sphere).
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

PI_REF = 3.1415926  # particle_system.py:623


# ------------------------------------------------------------------ loading
def _merge(vertices: np.ndarray, faces: np.ndarray):
    """Merges exactly equal vertices (first occurrence keeps its place)."""
    uniq, first, inverse = np.unique(vertices, axis=0, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")  # unique rows in first-occurrence order
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    return uniq[order], rank[inverse.reshape(-1)][faces]


def load_obj(path) -> tuple[np.ndarray, np.ndarray]:
    verts, faces = [], []
    for line in Path(path).read_text().splitlines():
        tok = line.split()
        if not tok or tok[0].startswith("#"):
            continue
        if tok[0] == "v":
            verts.append([float(t) for t in tok[1:4]])
        elif tok[0] == "f":
            idx = []
            for t in tok[1:]:
                k = int(t.split("/")[0])
                idx.append(k - 1 if k > 0 else len(verts) + k)
            for a in range(1, len(idx) - 1):  # fan
                faces.append([idx[0], idx[a], idx[a + 1]])
    v = np.asarray(verts, np.float64).reshape(-1, 3)
    f = np.asarray(faces, np.int64).reshape(-1, 3)
    if f.size and (f.min() < 0 or f.max() >= len(v)):
        raise ValueError(f"{path}: face index out of range")
    return v, f


def load_stl(path) -> tuple[np.ndarray, np.ndarray]:
    data = Path(path).read_bytes()
    if len(data) >= 84:
        n = struct.unpack_from("<I", data, 80)[0]
        if 84 + 50 * n == len(data):  # binary
            rec = np.frombuffer(data, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]),
                                count=n, offset=84)
            v = rec["v"].reshape(-1, 3).astype(np.float64)
            return v, np.arange(3 * n, dtype=np.int64).reshape(-1, 3)
    text = data.decode("ascii", errors="replace")
    v = [[float(t) for t in line.split()[1:4]] for line in text.splitlines() if line.strip().startswith("vertex")]
    if len(v) % 3:
        raise ValueError(f"{path}: ASCII STL with a partial facet")
    v = np.asarray(v, np.float64).reshape(-1, 3)
    return v, np.arange(len(v), dtype=np.int64).reshape(-1, 3)


def load_mesh(path) -> tuple[np.ndarray, np.ndarray]:
    """(vertices (n, 3) float64, faces (m, 3) int64) with duplicates merged."""
    ext = Path(path).suffix.lower()
    if ext == ".obj":
        v, f = load_obj(path)
    elif ext == ".stl":
        v, f = load_stl(path)
    else:
        raise ValueError(f"{path}: only .obj and .stl meshes are supported")
    if len(f) == 0:
        raise ValueError(f"{path}: no faces")
    return _merge(v, f)


# ---------------------------------------------------------------- placement
def rotation_matrix(angle: float, direction, point) -> np.ndarray:
    """4x4 rotation by angle (radians) about the axis `direction` through
    `point` (Rodrigues' formula)."""
    d = np.asarray(direction, np.float64)
    d = d / np.linalg.norm(d)
    c, s = np.cos(angle), np.sin(angle)
    R = c * np.eye(3) + s * np.array([[0, -d[2], d[1]], [d[2], 0, -d[0]], [-d[1], d[0], 0]]) \
        + (1.0 - c) * np.outer(d, d)
    M = np.eye(4)
    M[:3, :3] = R
    p = np.asarray(point, np.float64)
    M[:3, 3] = p - R @ p
    return M


def place(vertices: np.ndarray, rigid_body: dict) -> np.ndarray:
    """particle_system.py:618-628: scale, rotate about the vertex mean, translate."""
    v = vertices * np.asarray(rigid_body.get("scale", 1.0), np.float64)
    angle = rigid_body.get("rotationAngle", 0.0) / 360 * 2 * PI_REF
    axis = rigid_body.get("rotationAxis", [0.0, 0.0, 1.0])
    M = rotation_matrix(angle, axis, v.mean(axis=0))
    v = v @ M[:3, :3].T + M[:3, 3]
    return v + np.asarray(rigid_body.get("translation", [0.0, 0.0, 0.0]), np.float64)


# ------------------------------------------------------------ voxelisation
def subdivide_to_size(vertices: np.ndarray, faces: np.ndarray, max_edge: float, max_iter: int = 10) -> np.ndarray:
    """All vertices of the mesh after splitting, round by round, every face
    with an edge longer than max_edge into four at its edge midpoints."""
    allv = [vertices]
    v, f = vertices, faces
    for it in range(max_iter + 1):
        tri = v[f]
        edge = np.sqrt((np.diff(tri[:, [0, 1, 2, 0]], axis=1) ** 2).sum(axis=2))
        long_ = (edge > max_edge).any(axis=1)
        if not long_.any():
            return np.concatenate(allv)
        if it == max_iter:
            raise ValueError("mesh needs more than max_iter subdivisions at this pitch")
        f = f[long_]
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        mab = (v[a] + v[b]) / 2.0
        mbc = (v[b] + v[c]) / 2.0
        mca = (v[c] + v[a]) / 2.0
        n, m = len(v), len(f)
        v = np.concatenate([v, mab, mbc, mca])
        iab, ibc, ica = n + np.arange(m), n + m + np.arange(m), n + 2 * m + np.arange(m)
        f = np.concatenate([np.stack([a, iab, ica], 1), np.stack([iab, b, ibc], 1),
                            np.stack([ica, ibc, c], 1), np.stack([iab, ibc, ica], 1)])
        allv.append(v[n:])
    return np.concatenate(allv)


def voxelize_filled(vertices: np.ndarray, faces: np.ndarray, pitch: float) -> np.ndarray:
    """Centres of the surface voxels and the voxels they enclose, (k, 3)
    float64, lexicographic in the voxel index."""
    from scipy import ndimage
    pts = subdivide_to_size(vertices, faces, max_edge=pitch / 2.0)
    hit = np.unique(np.round(pts / pitch).astype(np.int64), axis=0)
    lo = hit.min(axis=0)
    shape = hit.max(axis=0) - lo + 1
    dense = np.zeros(tuple(shape), dtype=bool)
    dense[tuple((hit - lo).T)] = True
    dense = ndimage.binary_fill_holes(dense)
    return (np.argwhere(dense) + lo) * pitch


def rigid_body_points(rigid_body: dict, pitch: float) -> np.ndarray:
    """load_rigid_body (particle_system.py:616-639) for one `RigidBodies` entry."""
    v, f = load_mesh(rigid_body["geometryFile"])
    return voxelize_filled(place(v, rigid_body), f, pitch)
