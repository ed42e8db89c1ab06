"""ASCII PLY export with the reference's header and row format
(karman_vortex.py:122-214), read from the device buffers in one copy."""
from __future__ import annotations

from pathlib import Path

import numpy as np

from ._abi import MATERIAL_FLUID

_HEADER = (
    "ply\n"
    "format ascii 1.0\n"
    "element vertex {n}\n"
    "property float x\n"
    "property float y\n"
    "property float z\n"
    "property float vort_x\n"
    "property float vort_y\n"
    "property float vort_z\n"
    "property uchar red\n"
    "property uchar green\n"
    "property uchar blue\n"
    "property int object_id\n"
    "property uchar particle_type\n"
    "end_header\n"
)


def particle_types(ps, obj_id: np.ndarray) -> np.ndarray:
    """0 fluid block, 1 fluid emitter, 2 rigid block, 3 rigid body, 4 other
    (karman_vortex.py:159-179; later assignments win)."""
    t = np.full(obj_id.shape[0], 4, dtype=np.uint8)
    for ids, code in ((ps.obj_id_fluid_blocks, 0), (ps.obj_id_emitters, 1),
                      (ps.obj_id_rigid_blocks, 2), (ps.object_id_rigid_body, 3)):
        if ids:
            t[np.isin(obj_id, np.array(sorted(ids), dtype=obj_id.dtype))] = code
    return t


def write_ply(solver, cnt: int, ply_path: Path) -> Path | None:
    ps = solver.ps
    n = ps.particle_num[None]
    if n == 0:
        return None
    x = solver.x_temp[:n].cpu().numpy()
    vort = ps.vorticity[:n].cpu().numpy()
    color = ps.color[:n].cpu().numpy()
    obj_id = ps.object_id[:n].cpu().numpy()
    active = ps.is_active[:n].cpu().numpy().astype(bool)
    x, vort, color, obj_id = x[active], vort[active], color[active], obj_id[active]
    m = x.shape[0]
    if m == 0:
        return None
    if x.shape[1] == 2:
        x = np.concatenate([x, np.zeros((m, 1), dtype=x.dtype)], axis=1)
    ptype = particle_types(ps, obj_id)
    ply_path.mkdir(parents=True, exist_ok=True)
    path = ply_path / f"frame_{cnt:04}.ply"
    cols = [x[:, 0], x[:, 1], x[:, 2], vort[:, 0], vort[:, 1], vort[:, 2]]
    with open(path, "w") as f:
        f.write(_HEADER.format(n=m))
        rows = np.empty(m, dtype=object)
        fl = [np.char.mod("%.7f", c.astype(np.float64)) for c in cols]
        ints = [np.char.mod("%d", c) for c in (color[:, 0], color[:, 1], color[:, 2], obj_id, ptype)]
        parts = fl + ints
        line = parts[0]
        for p in parts[1:]:
            line = np.char.add(np.char.add(line, " "), p)
        f.write("\n".join(line.tolist()))
        f.write("\n")
    return path


# ------------------------------------------------------------------ PNG
# karman_vortex.py:38-121 draws the fluid particles coloured by the z
# vorticity of vorticity_vis (coolwarm, limits -40..40, alpha 0.6) and the
# particles of object 2 in #00C853, with matplotlib: a 3-D scatter seen from
# elevation 30 and azimuth -60 over the box [0,4]x[0,1]x[0,1] with aspect
# (4,1,1), or, in the 2-D variant kept in its comments, the xy plane over
# [0,4]x[0,1].  matplotlib is not a dependency here, so the same content is
# drawn with PIL: an orthographic view with those angles, each pixel showing
# the nearest particle that falls on it (fluid with alpha 0.6), on a
# transparent background.  It is not pixel-identical.
_COOLWARM = np.array([  # Moreland's diverging map at 0, 0.25, 0.5, 0.75, 1
    [59, 76, 192], [141, 176, 254], [221, 221, 221], [244, 154, 123], [180, 4, 38]], dtype=np.float64)
_SOLID_RGB = (0x00, 0xC8, 0x53)


def coolwarm(v: np.ndarray, vmin: float = -40.0, vmax: float = 40.0) -> np.ndarray:
    t = np.clip((np.asarray(v, np.float64) - vmin) / (vmax - vmin), 0.0, 1.0) * 4.0
    k = np.minimum(t.astype(np.int64), 3)
    w = (t - k)[:, None]
    return ((1.0 - w) * _COOLWARM[k] + w * _COOLWARM[k + 1]).round().astype(np.uint8)


def render_frame(x: np.ndarray, vort_z: np.ndarray, fluid: np.ndarray, solid: np.ndarray, width: int = 2048):
    """RGBA image (PIL) of one frame; x is (n, 2) or (n, 3)."""
    from PIL import Image
    x = np.asarray(x, np.float64)
    if x.shape[1] == 2:  # the xy plane over [0,4]x[0,1]
        u, w = x[:, 0] / 4.0, x[:, 1]
        height = width // 4
        depth = np.zeros(len(x))
    else:  # orthographic view, elevation 30, azimuth -60, box aspect (4,1,1)
        el, az = np.radians(30.0), np.radians(-60.0)
        p = (x - [2.0, 0.5, 0.5]) * [1.0, 1.0, 1.0]
        e = np.array([-np.sin(az), np.cos(az), 0.0])  # screen right
        f = np.array([np.cos(el) * np.cos(az), np.cos(el) * np.sin(az), np.sin(el)])  # towards the viewer
        up = np.cross(f, e)
        sx, sy, depth = p @ e, p @ up, p @ f
        half = 2.2  # half of the box diagonal in screen units, so the box fits
        u, w = (sx + half) / (2 * half), (sy + half / 2.5) / (2 * half / 2.5)
        height = int(width / 2.5)
    rgba = np.zeros((height, width, 4), np.uint8)
    cols = np.zeros((len(x), 4), np.uint8)
    cols[fluid, :3] = coolwarm(vort_z[fluid])
    cols[fluid, 3] = 153  # alpha 0.6
    cols[solid, :3] = _SOLID_RGB
    cols[solid, 3] = 255
    px = np.clip((u * (width - 1)).round().astype(np.int64), 0, width - 1)
    py = np.clip(((1.0 - w) * (height - 1)).round().astype(np.int64), 0, height - 1)
    sel = np.nonzero(fluid | solid)[0]
    sel = sel[np.argsort(-depth[sel], kind="stable")]  # near to far
    pix = py[sel] * width + px[sel]
    _, first = np.unique(pix, return_index=True)  # the nearest particle of each pixel
    k = sel[first]
    rgba.reshape(-1, 4)[py[k] * width + px[k]] = cols[k]
    return Image.fromarray(rgba, "RGBA")


def write_png(solver, cnt: int, image_path: Path) -> Path | None:
    ps = solver.ps
    n = ps.particle_num[None]
    if n == 0:
        return None
    x = solver.x_temp[:n].cpu().numpy()
    vort = solver.vorticity_vis[:n].cpu().numpy()
    material = ps.material[:n].cpu().numpy()
    obj_id = ps.object_id[:n].cpu().numpy()
    img = render_frame(x, vort[:, 2], material == MATERIAL_FLUID, obj_id == 2)
    image_path.mkdir(parents=True, exist_ok=True)
    path = image_path / f"vorticity_{cnt:04}.png"
    img.save(path)
    return path
