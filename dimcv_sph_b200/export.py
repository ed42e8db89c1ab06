"""Frame export with the reference's formats (karman_vortex.py:38-214).

PLY frames are written asynchronously: the fields are snapshotted on the
compute stream (a device-to-device copy, so later steps may overwrite them),
copied into pinned host buffers on a side stream, and formatted and written
by a worker thread, so the step loop does not wait for the file."""
from __future__ import annotations

import threading
from concurrent.futures import Future, ThreadPoolExecutor
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


def particle_types(obj_id: np.ndarray, fluid_blocks, emitters, rigid_blocks, rigid_bodies) -> np.ndarray:
    """0 fluid block, 1 fluid emitter, 2 rigid block, 3 rigid body, 4 other
    (karman_vortex.py:159-179; later assignments win)."""
    t = np.full(obj_id.shape[0], 4, dtype=np.uint8)
    for ids, code in ((fluid_blocks, 0), (emitters, 1), (rigid_blocks, 2), (rigid_bodies, 3)):
        if ids:
            t[np.isin(obj_id, np.array(sorted(ids), dtype=obj_id.dtype))] = code
    return t


def _object_sets(ps):
    return (frozenset(ps.obj_id_fluid_blocks), frozenset(ps.obj_id_emitters),
            frozenset(ps.obj_id_rigid_blocks), frozenset(ps.object_id_rigid_body))


def format_ply(x, vorticity, color, obj_id, is_active, object_sets) -> str | None:
    """The text of karman_vortex.py:136-214: the active particles' rows,
    `x y z vort_x vort_y vort_z r g b object_id particle_type`, floats as
    %.7f; None when no particle is active.  2-D positions get z = 0."""
    active = np.asarray(is_active).astype(bool)
    x, vort = np.asarray(x)[active], np.asarray(vorticity)[active]
    color, obj_id = np.asarray(color)[active], np.asarray(obj_id)[active]
    m = x.shape[0]
    if m == 0:
        return None
    if x.shape[1] == 2:
        x = np.concatenate([x, np.zeros((m, 1), dtype=x.dtype)], axis=1)
    ptype = particle_types(obj_id, *object_sets)
    cols = [x[:, 0], x[:, 1], x[:, 2], vort[:, 0], vort[:, 1], vort[:, 2]]
    parts = [np.char.mod("%.7f", c.astype(np.float64)) for c in cols]
    parts += [np.char.mod("%d", c) for c in (color[:, 0], color[:, 1], color[:, 2], obj_id, ptype)]
    line = parts[0]
    for p in parts[1:]:
        line = np.char.add(np.char.add(line, " "), p)
    return _HEADER.format(n=m) + "\n".join(line.tolist()) + "\n"


class AsyncPlyWriter:
    """PLY frames of one particle system, written off the step loop.

    `submit` records the frame and returns at once; `flush` waits for every
    frame and raises the first error.  Two buffer sets are kept, so a third
    frame in flight waits for the oldest one to be written."""

    FIELDS = ("x_temp", "vorticity", "color", "object_id", "is_active")

    def __init__(self, ps, slots: int = 2):
        import torch
        self.ps = ps
        self.side = torch.cuda.Stream(ps.device)
        self.pool = ThreadPoolExecutor(max_workers=1, thread_name_prefix="ply")
        self.slots = [None] * slots
        self.next = 0
        self.futures: list[Future] = []
        self.lock = threading.Lock()

    def _sources(self, solver):
        ps = self.ps
        return {"x_temp": solver.x_temp, "vorticity": ps.vorticity, "color": ps.color,
                "object_id": ps.object_id, "is_active": ps.is_active}

    def _slot(self, src, n):
        import torch
        k = self.next
        self.next = (k + 1) % len(self.slots)
        slot = self.slots[k]
        if slot is not None and slot["future"] is not None:
            slot["future"].result()  # the worker is done with these buffers
        if slot is None or slot["cap"] < n:
            cap = max(n, 1)
            slot = {"cap": cap, "future": None, "dev": {}, "pin": {}}
            for name, t in src.items():
                shape = (cap,) + tuple(t.shape[1:])
                slot["dev"][name] = torch.empty(shape, dtype=t.dtype, device=t.device)
                slot["pin"][name] = torch.empty(shape, dtype=t.dtype, pin_memory=True)
            self.slots[k] = slot
        return slot

    def submit(self, solver, cnt: int, ply_path: Path) -> Path | None:
        import torch
        ps = self.ps
        n = ps.particle_num[None]
        if n == 0:
            return None
        src = self._sources(solver)
        slot = self._slot(src, n)
        with torch.cuda.stream(ps.stream):
            for name, t in src.items():
                slot["dev"][name][:n].copy_(t[:n])
            snap = torch.cuda.Event()
            snap.record(ps.stream)
        self.side.wait_event(snap)
        with torch.cuda.stream(self.side):
            for name in src:
                slot["pin"][name][:n].copy_(slot["dev"][name][:n], non_blocking=True)
            done = torch.cuda.Event()
            done.record(self.side)
        ply_path = Path(ply_path)
        ply_path.mkdir(parents=True, exist_ok=True)
        path = ply_path / f"frame_{cnt:04}.ply"
        sets = _object_sets(ps)
        fut = self.pool.submit(self._write, done, slot, n, sets, path)
        slot["future"] = fut
        with self.lock:
            self.futures.append(fut)
        return path

    @staticmethod
    def _write(done, slot, n, sets, path: Path) -> Path | None:
        done.synchronize()
        a = {k: v[:n].numpy() for k, v in slot["pin"].items()}
        text = format_ply(a["x_temp"], a["vorticity"], a["color"], a["object_id"], a["is_active"], sets)
        if text is None:
            return None
        with open(path, "w") as f:
            f.write(text)
        return path

    def flush(self):
        with self.lock:
            futs, self.futures = self.futures, []
        for f in futs:
            f.result()


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
