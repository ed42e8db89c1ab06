"""KarmanVortexSolver with the reference's step / substep order
(karman_vortex.py:8-36, 122-242).  The obstacle is configurable
(`cylinderCenter`, `cylinderRadius`, `cylinderObjectId`); the defaults are the
reference's hard-coded (0.65, 0.5, 0.5), 0.1 and object 2."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import torch

from .dimcv_sph import DIMCVSPHSolver


class KarmanVortexSolver(DIMCVSPHSolver):
    def __init__(self, particle_system):
        super().__init__(particle_system)
        g = self.ps.cfg.get_cfg
        self.circle_pos = np.array(g("cylinderCenter") or [0.65, 0.5, 0.5], dtype=np.float64)
        self.circle_radius = float(g("cylinderRadius") if g("cylinderRadius") is not None else 0.1)
        self.cylinder_object_id = int(g("cylinderObjectId") if g("cylinderObjectId") is not None else 2)
        # "cylinder" (x-y distance, the reference) or "sphere" (3-D distance)
        self.obstacle_shape = g("obstacleShape") or "cylinder"
        self.compute_vis = bool(g("computeVis") if g("computeVis") is not None else True)
        self.bounce_back = bool(g("bounceBackBoundary"))
        self.init_cylinder()

    def init_cylinder(self):
        """karman_vortex.py:27-36: object-2 particles farther than the radius
        from the cylinder axis (x-y distance) move to the origin and become
        inactive (update_activity re-activates solids, as in the reference)."""
        ps = self.ps
        n = ps.particle_num[None]
        if n == 0:
            return
        x = ps.x[:n]
        oid = ps.object_id[:n]
        cx = torch.tensor(np.float32(self.circle_pos[0]), device=ps.device)
        cy = torch.tensor(np.float32(self.circle_pos[1]), device=ps.device)
        dx = x[:, 0] - cx
        dy = x[:, 1] - cy
        d2 = dx * dx + dy * dy
        if self.obstacle_shape == "sphere" and ps.dim == 3:
            dz = x[:, 2] - torch.tensor(np.float32(self.circle_pos[2]), device=ps.device)
            d2 = d2 + dz * dz
        far = (oid == self.cylinder_object_id) & (torch.sqrt(d2) > np.float32(self.circle_radius))
        x[far] = 0.0
        ps.is_active[:n][far] = 0

    def step(self):  # karman_vortex.py:216-230
        self.dump_num_particles_each_emitters_ti2np()
        if self.cnt % self.emit_interval == 0:
            self.emit_particle()
            self.dump_num_particles_each_emitters_np2ti()
        self.cnt += 1
        self.ps.initialize_particle_system()
        self.compute_moving_boundary_volume()
        self.substep()
        if self.bounce_back:  # karman_vortex.py:226-230
            if self.ps.dim == 2:
                self.enforce_boundary_2D(self.ps.material_fluid)
            else:
                self.enforce_boundary_3D(self.ps.material_fluid)

    def substep(self):  # karman_vortex.py:232-242
        self.compute_densities()
        self.compute_DFSPH_factor()
        self.divergence_solve()
        self.compute_non_pressure_forces()
        self.dimcv()
        self.predict_velocity()
        self.pressure_solve()
        if self.compute_vis:
            self.copy_x_temp()
            self.compute_vorticity_vis()
        self.advect()

    def export_png(self, cnt, image_path):
        """vorticity_{cnt:04}.png of karman_vortex.py:38-121 (same view, colour
        map and limits), drawn with PIL instead of matplotlib."""
        from .export import write_png
        return write_png(self, cnt, Path(image_path))

    def export_ply(self, cnt, ply_path):
        """ASCII PLY with the reference's header and row format
        (karman_vortex.py:122-214).  Asynchronous: returns the file's path at
        once; the file is complete after flush_exports()."""
        if getattr(self, "_ply_writer", None) is None:
            from .export import AsyncPlyWriter
            self._ply_writer = AsyncPlyWriter(self.ps)
        return self._ply_writer.submit(self, cnt, Path(ply_path))

    def flush_exports(self):
        """Waits until every PLY frame submitted by export_ply is written."""
        if getattr(self, "_ply_writer", None) is not None:
            self._ply_writer.flush()
