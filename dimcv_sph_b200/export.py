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
