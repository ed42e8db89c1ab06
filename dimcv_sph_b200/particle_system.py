"""ParticleSystem with the reference's interface (particle_system.py:10-696),
holding particle state as torch CUDA tensors and running the neighbour grid
through libdimcv.

Differences a caller can see, all deliberate:
  * fields are torch tensors (``ps.x`` is a (capacity, dim) view of a
    padded buffer), scalars such as ``ps.particle_num[None]`` read the device
    counters (a synchronisation, as a Taichi scalar read is);
  * ``initialize_particle_system`` runs update_activity and one fused
    partition + cell sort (a stable radix sort on Morton cell keys) that
    writes into a second buffer set, then swaps the sets — the tensors behind
    ``ps.x`` etc. change identity at every rebuild;
  * ``grid_ids`` holds the Morton cell key (the reference stores the
    row-major flat index); neighbour sets are the same;
  * mesh rigid bodies are voxelised by ``mesh.py`` (OBJ / STL, a restatement
    of trimesh's subdivide voxeliser and hole fill, as trimesh is not a
    dependency); the pressure solve's reaction on dynamic rigid particles is
    gathered per particle in a fixed order (the reference adds it with
    unordered atomics); GGUI buffers are not supported: no drawing path.
"""
from __future__ import annotations

import ctypes as C
from functools import reduce

import numpy as np
import torch

from .mesh import rigid_body_points
from . import _lib
from ._abi import MATERIAL_FLUID, MATERIAL_SOLID, DvCounters
from .fields import particle_fields, solver_fields
from .params import Options, make_params


class Scalar:
    """0-d device scalar with the Taichi `field[None]` access form."""

    def __init__(self, getter, setter=None):
        self._get = getter
        self._set = setter

    def __getitem__(self, key):
        return self._get()

    def __setitem__(self, key, value):
        if self._set is None:
            raise AttributeError("read-only scalar")
        self._set(value)

    def __repr__(self):
        return f"Scalar({self._get()!r})"


class ParticleSystem:
    material_solid = MATERIAL_SOLID
    material_fluid = MATERIAL_FLUID

    def __init__(self, config, GGUI=False, device=None, options: Options | None = None,
                 capacity: int | None = None, verbose: bool = False, grid_num=None):
        self.cfg = config
        self.GGUI = GGUI  # accepted for signature compatibility; nothing is drawn
        self.verbose = verbose
        self.device = torch.device(device or "cuda")
        if self.device.type != "cuda":
            raise RuntimeError("ParticleSystem runs on a CUDA device only (no CPU fallback)")
        self.lib = _lib.load()
        g = config.get_cfg
        self.domain_start = np.array(g("domainStart"))
        self.domain_end = np.array(g("domainEnd"))
        self.domain_size = self.domain_end - self.domain_start
        self.window_res = g("windowRes")
        self.dim = len(self.domain_size)
        assert self.dim > 1
        self.simulation_method = g("simulationMethod")
        self.particle_radius = g("particleRadius")
        self.particle_diameter = 2 * self.particle_radius
        self.support_radius = self.particle_radius * 4.0
        self.inv_support_radius = 1.0 / self.support_radius
        self.m_V0 = 0.8 * self.particle_diameter ** self.dim
        self.grid_size = self.support_radius
        self.inv_grid_size = 1.0 / self.grid_size
        self.grid_num = np.ceil(self.domain_size / self.grid_size).astype(int)
        self.flattened_grid_num = int(reduce(lambda a, b: a * b, self.grid_num))
        self.padding = self.grid_size
        if verbose:
            print("grid num: ", self.grid_num)

        self.object_collection = dict()
        self.object_id_rigid_body = set()
        self.obj_id_emitters = set()
        self.obj_id_fluid_blocks = set()
        self.obj_id_rigid_blocks = set()

        fluid_blocks = config.get_fluid_blocks()
        fluid_particle_num = 0
        for fluid in fluid_blocks:
            n = self._block_count(fluid)
            fluid["particleNum"] = n
            self.object_collection[fluid["objectId"]] = fluid
            fluid_particle_num += n
        rigid_blocks = config.get_rigid_blocks()
        rigid_particle_num = 0
        for rigid in rigid_blocks:
            n = self._block_count(rigid)
            rigid["particleNum"] = n
            self.object_collection[rigid["objectId"]] = rigid
            self.obj_id_rigid_blocks.add(rigid["objectId"])
            rigid_particle_num += n
        # mesh rigid bodies (particle_system.py:90-97, 616-639), static only
        rigid_bodies = config.get_rigid_bodies() or []
        for body in rigid_bodies:
            if self.dim != 3:
                raise ValueError("mesh rigid bodies need a 3-D scene")
            pts = rigid_body_points(body, 2 * g("particleRadius"))
            body["particleNum"] = int(pts.shape[0])
            body["voxelizedPoints"] = pts
            self.object_collection[body["objectId"]] = body
            rigid_particle_num += int(pts.shape[0])
        self.fluid_emitters = config.get_fluid_emitters()
        self.num_emitters = 0
        for emitter in self.fluid_emitters:
            self.obj_id_emitters.add(emitter["objectId"])
            self.num_emitters += 1
            emitter["particleNum"] = 0
            self.object_collection[emitter["objectId"]] = emitter
        self.particle_max_num = fluid_particle_num + rigid_particle_num
        self.reserved_capacity = g("reservedCapacity")
        if self.reserved_capacity is not None:
            self.particle_max_num += self.reserved_capacity
        if capacity is not None:
            self.particle_max_num = max(int(capacity), self.particle_max_num)
        self.num_rigid_bodies = len(rigid_blocks) + len(rigid_bodies)

        # device state: two particle field sets (the grid build gathers from one
        # into the other) and the index-stable solver fields
        self.options = options or Options.from_config(config)
        self.params = make_params(config, self.options)
        if grid_num is not None:  # a larger cell grid (same Morton layout as a scene batch)
            for d in range(self.dim):
                if int(grid_num[d]) < self.params.grid_num[d]:
                    raise ValueError("grid_num may only enlarge the cell grid")
                self.params.grid_num[d] = int(grid_num[d])
        cap = int(self.particle_max_num)
        self._sets = [particle_fields(cap, self.dim, self.device), particle_fields(cap, self.dim, self.device)]
        self._cur = 0
        self.solver_buf = solver_fields(cap, self.dim, self.device)
        self.stream = torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            self.ctx = self.lib.dv_create(C.byref(self.params), cap, C.c_void_p(self.stream.cuda_stream))
        if not self.ctx:
            raise _lib.DimcvError(f"dv_create failed: {self.lib.dv_last_error(None).decode()}")
        self.cnt = 0

        for fluid in fluid_blocks:
            self.obj_id_fluid_blocks.add(fluid["objectId"])
            offset = np.array(fluid["translation"])
            start = np.array(fluid["start"]) + offset
            end = np.array(fluid["end"]) + offset
            scale = np.array(fluid["scale"])
            self.add_cube(object_id=fluid["objectId"], lower_corner=start,
                          cube_size=(end - start) * scale, velocity=fluid["velocity"],
                          density=fluid["density"], is_dynamic=1, color=fluid["color"],
                          material=MATERIAL_FLUID, exclude=self._exclusion(fluid))
        for rigid in rigid_blocks:
            offset = np.array(rigid["translation"])
            start = np.array(rigid["start"]) + offset
            end = np.array(rigid["end"]) + offset
            scale = np.array(rigid["scale"])
            self.add_cube(object_id=rigid["objectId"], lower_corner=start,
                          cube_size=(end - start) * scale, velocity=rigid["velocity"],
                          density=rigid["density"], is_dynamic=rigid["isDynamic"],
                          color=rigid["color"], material=MATERIAL_SOLID,
                          exclude=self._exclusion(rigid))
        for body in rigid_bodies:  # particle_system.py:276-303
            self.object_id_rigid_body.add(body["objectId"])
            n = body["particleNum"]
            if n == 0:
                continue
            dyn = 1 if body.get("isDynamic") else 0
            vel = np.asarray(body["velocity"], np.float32)[:self.dim] if dyn else np.zeros(self.dim, np.float32)
            pos = np.asarray(body["voxelizedPoints"], np.float32)[:, :self.dim]
            self.add_particles(body["objectId"], n, pos, np.tile(vel, (n, 1)),
                               np.full(n, body["density"], np.float32), np.zeros(n, np.float32),
                               np.full(n, MATERIAL_SOLID, np.int32), np.full(n, dyn, np.int32),
                               np.tile(np.asarray(body["color"], np.int32), (n, 1)))
        # dynamic rigid particles (rigid blocks or bodies with isDynamic): no
        # shape matching, as in the reference, where it is never called; the
        # pressure solve adds their reaction (dimcv_sph.py:540-549)
        self.has_dynamic_rigid = any(bool(r.get("isDynamic")) for r in list(rigid_blocks) + list(rigid_bodies))
        if self.has_dynamic_rigid:
            _lib.check(self.ctx, self.lib.dv_set_dynamic_rigid(self.ctx, 1), "dv_set_dynamic_rigid")
        if verbose:
            print(f"Current particle num: {self.particle_num[None]}, Particle max num: {self.particle_max_num}")

    def __del__(self):
        ctx = getattr(self, "ctx", None)
        if ctx:
            try:
                self.lib.dv_destroy(ctx)
            except Exception:
                pass
            self.ctx = None

    # ------------------------------------------------------------ geometry
    def _block_count(self, block) -> int:
        start = np.array(block["start"]) + np.array(block.get("translation", [0.0] * self.dim))
        end = np.array(block["end"]) + np.array(block.get("translation", [0.0] * self.dim))
        scale = np.array(block.get("scale", [1] * self.dim))
        pts = self._lattice(start, (end - start) * scale, self._exclusion(block))
        return pts.shape[0]

    def _exclusion(self, block):
        """New keys: a block may carve out disks/balls ("exclude": [{"center",
        "radius"}]) so a fluid lattice does not overlap an obstacle, or keep
        only the lattice points inside one ("keepInside": {"center", "radius"})
        to build a solid disk/ball directly."""
        out = []
        for e in block.get("exclude") or []:
            out.append((np.array(e["center"], dtype=np.float64)[: self.dim], float(e["radius"]), False))
        k = block.get("keepInside")
        if k:
            out.append((np.array(k["center"], dtype=np.float64)[: self.dim], float(k["radius"]), True))
        return out or None

    def compute_cube_particle_num(self, start, end):  # particle_system.py:641-645
        num_dim = [np.arange(start[i], end[i], self.particle_diameter) for i in range(self.dim)]
        return reduce(lambda a, b: a * b, [len(n) for n in num_dim])

    def _lattice(self, lower_corner, cube_size, exclude=None) -> np.ndarray:
        num_dim = [np.arange(lower_corner[i], lower_corner[i] + cube_size[i], self.particle_diameter)
                   for i in range(self.dim)]
        pos = np.array(np.meshgrid(*num_dim, sparse=False, indexing="ij"), dtype=np.float32)
        pos = pos.reshape(self.dim, -1).transpose().copy()
        if exclude:
            keep = np.ones(pos.shape[0], dtype=bool)
            for center, radius, inside in exclude:
                d = pos.astype(np.float64) - center[None, :]
                dist = np.sqrt((d * d).sum(axis=1))
                keep &= (dist <= radius) if inside else (dist > radius)
            pos = pos[keep]
        return pos

    # ------------------------------------------------------------ particles
    def add_cube(self, object_id, lower_corner, cube_size, material, is_dynamic, color=(0, 0, 0),
                 density=None, pressure=None, velocity=None, exclude=None):
        """particle_system.py:647-696 (optionally minus excluded disks/balls)."""
        pos = self._lattice(np.asarray(lower_corner), np.asarray(cube_size), exclude)
        n = pos.shape[0]
        if velocity is None:
            vel = np.zeros_like(pos)
        else:
            vel = np.tile(np.asarray(velocity, dtype=np.float32)[: self.dim], (n, 1))
        self._add(object_id, pos, vel, 1000.0 if density is None else density,
                  0.0 if pressure is None else pressure, material, is_dynamic, color)
        return n

    def add_particles(self, object_id, new_particles_num, new_particles_positions,
                      new_particles_velocity, new_particle_density, new_particle_pressure,
                      new_particles_material, new_particles_is_dynamic, new_particles_color):
        """particle_system.py:334-380; per-particle arrays, grouped into runs of
        equal (density, pressure, material, is_dynamic, color)."""
        n = int(new_particles_num)
        pos = np.asarray(new_particles_positions, dtype=np.float32).reshape(n, self.dim)
        vel = np.asarray(new_particles_velocity, dtype=np.float32).reshape(n, self.dim)
        keys = np.stack([np.asarray(new_particle_density, np.float64),
                         np.asarray(new_particle_pressure, np.float64),
                         np.asarray(new_particles_material, np.float64),
                         np.asarray(new_particles_is_dynamic, np.float64),
                         *np.asarray(new_particles_color, np.float64).reshape(n, 3).T], axis=1)
        start = 0
        for i in range(1, n + 1):
            if i == n or not np.array_equal(keys[i], keys[start]):
                k = keys[start]
                self._add(object_id, pos[start:i], vel[start:i], k[0], k[1], int(k[2]), int(k[3]),
                          (int(k[4]), int(k[5]), int(k[6])))
                start = i

    def _add(self, object_id, pos, vel, density, pressure, material, is_dynamic, color):
        n = int(pos.shape[0])
        if n == 0:
            return
        d_pos = torch.from_numpy(np.ascontiguousarray(pos, dtype=np.float32)).to(self.device)
        d_vel = torch.from_numpy(np.ascontiguousarray(vel, dtype=np.float32)).to(self.device)
        col = list(color) + [0, 0, 0]
        rc = self.lib.dv_add_particles(
            self.ctx, C.byref(self.fields_struct), C.c_void_p(d_pos.data_ptr()),
            C.c_void_p(d_vel.data_ptr()), n, int(object_id), float(np.float32(density)),
            float(np.float32(pressure)), int(material), int(bool(is_dynamic)), int(col[0]),
            int(col[1]), int(col[2]), float(np.float32(self.m_V0)))
        _lib.check(self.ctx, rc, "dv_add_particles")
        # keep the staging tensors alive until the copy kernel has run
        self._staging = (d_pos, d_vel)

    # --------------------------------------------------------- grid rebuild
    def update_activity(self):  # particle_system.py:413-427
        _lib.check(self.ctx, self.lib.dv_update_activity(self.ctx, C.byref(self.fields_struct)),
                   "dv_update_activity")

    def counting_sort(self):
        """particle_partition + update_grid_id + prefix sum + counting_sort
        (particle_system.py:429-553) as one fused stable sort."""
        src = self._sets[self._cur]
        dst = self._sets[1 - self._cur]
        _lib.check(self.ctx, self.lib.dv_grid_build(self.ctx, C.byref(src.struct), C.byref(dst.struct)),
                   "dv_grid_build")
        self._cur = 1 - self._cur

    def particle_partition(self):
        """Fused into counting_sort (inactive particles sort behind every cell)."""

    def update_grid_id(self):
        """Fused into counting_sort (the cell keys are computed there)."""

    def initialize_particle_system(self):  # particle_system.py:555-560
        self.update_activity()
        self.counting_sort()

    def permutation(self) -> np.ndarray:
        """perm[p] = slot before the last rebuild of the particle now at p."""
        n = self.particle_num[None]
        out = np.zeros(max(n, 1), dtype=np.int32)
        rc = self.lib.dv_get_permutation(self.ctx, out.ctypes.data_as(C.POINTER(C.c_int32)), n)
        _lib.check(self.ctx, rc, "dv_get_permutation")
        return out[:n]

    def neighbor_lists(self):
        """CSR of for_all_neighbors (particle_system.py:562-586) in visit order:
        (offsets int64 [n+1], neighbours int32 [pairs]) on the device."""
        n = self.particle_num[None]
        off = torch.zeros(n + 1, dtype=torch.int64, device=self.device)
        total = self.lib.dv_neighbor_lists(self.ctx, C.byref(self.fields_struct),
                                           C.c_void_p(off.data_ptr()), None, 0)
        _lib.check(self.ctx, total, "dv_neighbor_lists")
        nbr = torch.zeros(max(total, 1), dtype=torch.int32, device=self.device)
        total = self.lib.dv_neighbor_lists(self.ctx, C.byref(self.fields_struct),
                                           C.c_void_p(off.data_ptr()), C.c_void_p(nbr.data_ptr()), total)
        _lib.check(self.ctx, total, "dv_neighbor_lists")
        return off, nbr[:total]

    def stored_neighbor_lists(self):
        """The lists the sweeps read, as the last grid build stored them:
        (offsets int64 [n+1], neighbours int32 [pairs]) on the device.  Rows
        of static solids are empty (no sweep of the step walks them)."""
        n = self.particle_num[None]
        off = torch.zeros(n + 1, dtype=torch.int32, device=self.device)
        total = self.lib.dv_stored_lists(self.ctx, C.c_void_p(off.data_ptr()), None, 0)
        _lib.check(self.ctx, total, "dv_stored_lists")
        nbr = torch.zeros(max(total, 1), dtype=torch.int32, device=self.device)
        total = self.lib.dv_stored_lists(self.ctx, None, C.c_void_p(nbr.data_ptr()), total)
        _lib.check(self.ctx, total, "dv_stored_lists")
        return off.to(torch.int64), nbr[:total]

    # ----------------------------------------------------------- counters
    def counters(self) -> dict:
        c = DvCounters()
        _lib.check(self.ctx, self.lib.dv_get_counters(self.ctx, C.byref(c)), "dv_get_counters")
        return c.as_dict()

    def set_counts(self, n: int, n_fluid: int, n_solid: int):
        _lib.check(self.ctx, self.lib.dv_set_counts(self.ctx, n, n_fluid, n_solid), "dv_set_counts")

    @property
    def particle_num(self):
        return Scalar(lambda: self.counters()["n"])

    @property
    def fluid_particle_num(self):
        return Scalar(lambda: self.counters()["n_fluid"])

    @property
    def solid_particle_num(self):
        return Scalar(lambda: self.counters()["n_solid"])

    @property
    def num_particles_each_emitter(self):
        """Active fluid particles per emitter object id (computed on demand)."""
        n = self.particle_num[None]
        oid = self.object_id[:n]
        mat = self.material[:n]
        act = self.is_active[:n]
        out = {}
        for obj in sorted(self.obj_id_emitters):
            out[obj] = int(((oid == obj) & (mat == MATERIAL_FLUID) & (act == 1)).sum().item())
        return out

    # ------------------------------------------------------------- fields
    @property
    def fields(self):
        return self._sets[self._cur]

    @property
    def fields_struct(self):
        return self._sets[self._cur].struct

    def _vec(self, name):
        return self._sets[self._cur][name][:, : self.dim]

    x = property(lambda self: self._vec("x"))
    x_0 = property(lambda self: self._vec("x0"))
    v = property(lambda self: self._vec("v"))
    acceleration = property(lambda self: self._vec("acceleration"))
    vorticity = property(lambda self: self._sets[self._cur]["vorticity"][:, :3])
    color = property(lambda self: self._sets[self._cur]["color"][:, :3])
    m_V = property(lambda self: self._sets[self._cur]["m_V"])
    m = property(lambda self: self._sets[self._cur]["m"])
    density = property(lambda self: self._sets[self._cur]["density"])
    pressure = property(lambda self: self._sets[self._cur]["pressure"])
    dfsph_factor = property(lambda self: self._sets[self._cur]["dfsph_factor"])
    density_adv = property(lambda self: self._sets[self._cur]["density_adv"])
    life_time = property(lambda self: self._sets[self._cur]["life_time"])
    material = property(lambda self: self._sets[self._cur]["material"])
    object_id = property(lambda self: self._sets[self._cur]["object_id"])
    grid_ids = property(lambda self: self._sets[self._cur]["grid_ids"])
    is_dynamic = property(lambda self: self._sets[self._cur]["is_dynamic"])
    is_active = property(lambda self: self._sets[self._cur]["is_active"])
    is_sample = property(lambda self: self._sets[self._cur]["is_sample"])
    vorticity_vis = property(lambda self: self.solver_buf["vorticity_vis"][:, :3])

    def snapshot(self, n: int | None = None) -> dict:
        """Host copies of every field for the first n slots (numpy)."""
        if n is None:
            n = self.particle_num[None]
        out = {k: t[:n].cpu().numpy().copy() for k, t in self.fields.t.items()}
        out.update({"solver." + k: t[:n].cpu().numpy().copy() for k, t in self.solver_buf.t.items()})
        return out

    def build_solver(self):  # particle_system.py:309-314
        if self.simulation_method == 0 or self.simulation_method is None:
            from .karman_vortex import KarmanVortexSolver
            return KarmanVortexSolver(self)
        raise NotImplementedError(f"Solver type {self.simulation_method} has not been implemented.")
