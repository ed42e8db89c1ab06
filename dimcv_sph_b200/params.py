"""dv_params from a scene configuration.

Every f32 constant is derived the way the reference's Taichi kernels see it:
Python-scope arithmetic happens in float64 and is rounded to f32 once where
it enters a kernel; values that the reference first stores in a Taichi local
(an f32 variable) are rounded there and combined in f32.  The cited lines are
the reference expressions each constant stands for.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from ._abi import DV_KERNEL_BLOB3D, DV_KERNEL_REF2D, DvParams


def f32(x: float) -> float:
    return float(np.float32(x))


def f32_pow_int(base: float, n: int) -> float:
    """Taichi lowers `f32 ** int` to exponentiation by squaring in f32."""
    res = np.float32(1.0)
    b = np.float32(base)
    while n > 0:
        if n & 1:
            res = np.float32(res * b)
        b = np.float32(b * b)
        n >>= 1
    return float(res)


def sqrt_limits(h: float) -> tuple[float, float]:
    """(lo, hi): lo = smallest f32 t with sqrtf(t) >= h, hi = largest f32 t
    with sqrtf(t) <= h.  Since IEEE sqrt is monotone, sqrtf(r2) < h <=> r2 < lo
    and sqrtf(r2) > h <=> r2 > hi."""
    h32 = np.float32(h)
    t = np.float32(h32 * h32)
    # smallest t with sqrt(t) >= h
    lo = t
    while np.sqrt(lo) >= h32:
        lo = np.nextafter(lo, np.float32(0))
    while np.sqrt(lo) < h32:
        lo = np.nextafter(lo, np.float32(np.inf))
    hi = t
    while np.sqrt(hi) <= h32:
        hi = np.nextafter(hi, np.float32(np.inf))
    while np.sqrt(hi) > h32:
        hi = np.nextafter(hi, np.float32(0))
    return float(lo), float(hi)


@dataclass
class Options:
    """Switches with no counterpart in the reference (defaults = reference)."""
    skip_cell0: bool = True          # particle_system.py:581-583 quirk
    cell_origin_offset: bool = False  # cell = int((x - domainStart)/h) instead of int(x/h)
    kernel: str = "ref2d"            # "ref2d" (dimcv_sph.py:649-719) | "blob3d"
    blob_delta: float | None = None  # regularisation radius of blob3d (default: particle radius)
    compensated: bool = False        # compensated f32 accumulation in the N-body sums
    periodic: bool = False           # every axis wraps; minimum-image distances
    extra: dict = field(default_factory=dict)

    @classmethod
    def from_config(cls, cfg) -> "Options":
        o = cls()
        g = cfg.get_cfg
        if g("skipCell0") is not None:
            o.skip_cell0 = bool(g("skipCell0"))
        if g("cellOriginOffset") is not None:
            o.cell_origin_offset = bool(g("cellOriginOffset"))
        if g("kernel3D") is not None:
            o.kernel = "blob3d" if g("kernel3D") else "ref2d"
        if g("blobDelta") is not None:
            o.blob_delta = float(g("blobDelta"))
        if g("compensated") is not None:
            o.compensated = bool(g("compensated"))
        if g("periodic") is not None:
            o.periodic = bool(g("periodic"))
        return o


def make_params(cfg, options: Options | None = None) -> DvParams:
    g = cfg.get_cfg
    if g("domainStart") is None or g("domainEnd") is None:
        seg = " (a SegmentConfiguration scene of the reference's vortex-segment solver, " \
              "run_segment_simulation.py, which this library does not implement)" \
            if "SegmentConfiguration" in getattr(cfg, "config", {}) else ""
        raise ValueError("the scene has no Configuration.domainStart / domainEnd, which the SPH particle "
                         f"system needs (particle_system.py:17-20){seg}")
    o = options or Options.from_config(cfg)
    domain_start = np.array(g("domainStart"), dtype=np.float64)  # particle_system.py:17
    domain_end = np.array(g("domainEnd"), dtype=np.float64)      # :20
    domain_size = domain_end - domain_start                      # :22
    dim = len(domain_size)                                       # :26
    if dim not in (2, 3):
        raise ValueError(f"dim must be 2 or 3, got {dim}")
    r = float(g("particleRadius"))                               # :41
    diameter = 2 * r                                             # :43
    support = r * 4.0                                            # :44
    inv_support = 1.0 / support                                  # :45
    m_V0 = 0.8 * diameter ** dim                                 # :46
    grid_num = np.ceil(domain_size / support).astype(int)        # :54

    p = DvParams()
    p.dim = dim
    for d in range(3):
        p.grid_num[d] = int(grid_num[d]) if d < dim else 1
        p.domain_start[d] = f32(domain_start[d]) if d < dim else 0.0
        p.domain_end[d] = f32(domain_end[d]) if d < dim else 0.0
    p.grid_size = f32(support)                                   # pos / grid_size (:383)
    p.support_radius = f32(support)                              # .norm() < support_radius (:585)
    h32 = f32(inv_support)                                       # h = inv_support_radius, f32 local (sph_base.py:26,48)
    p.inv_support_radius = h32
    p.nbr_r2_limit, p.far_r2_limit = sqrt_limits(p.support_radius)
    k_dim = {2: 1.8189, 3: 2.5465}[dim]                          # sph_base.py:31-34
    hd = f32_pow_int(h32, dim)                                   # h ** dim (sph_base.py:35)
    p.kW = f32(np.float32(k_dim) * np.float32(hd))               # k *= h ** dim
    p.kW2 = f32(np.float32(p.kW) * np.float32(2.0))              # k * 2 (sph_base.py:43)
    p.kG = f32(np.float32(np.float32(6.0) * np.float32(k_dim)) * np.float32(hd))  # 6. * k * h**dim (:57)
    p.grad_r_min = f32(1e-5)                                     # sph_base.py:61
    density0 = float(g("density0")) if g("density0") is not None else 1000.0
    p.density0 = f32(density0)                                   # sph_base.py:16-17
    dt = f32(g("timeStepSize"))                                  # dimcv_sph.py:13 (f32 field)
    p.dt = dt
    inv_dt = 1.0 / dt                                            # dimcv_sph.py:27 (Python float)
    p.inv_dt = f32(inv_dt)
    p.inv_dt2 = f32(1.0 / (dt * dt))                             # :28
    grav = list(g("gravitation") or [0.0] * dim)                 # sph_base.py:12
    for d in range(3):
        p.gravity[d] = f32(grav[d]) if d < dim else 0.0
    viscosity = 1e-3                                             # sph_base.py:14
    d_int = 2 * (dim + 2)                                        # dimcv_sph.py:170 (i32 local)
    p.visc_coef = f32(np.float32(d_int) * np.float32(viscosity))  # d * self.viscosity
    p.visc_h2 = f32(0.01 * support ** 2)                         # :178
    p.m_eps = f32(1e-5)                                          # :24
    p.factor_min = f32(1e-6)                                     # :102
    p.eta_div = inv_dt * 0.1 * 0.01 * density0                   # :389
    p.eta_p = 0.05 * 0.01 * density0                             # :611
    p.max_iter_div = int(g("maxIterationsV") or 100)             # :22
    p.max_iter_p = int(g("maxIterations") or 100)                # :23
    p.neighbor_min = 20 if dim == 3 else 7                       # :351-356
    area = g("divergenceTransitArea")                            # :63-64
    if area is not None:
        p.has_transit = 1
        p.transit_a0 = f32(area[0])
        p.transit_span = f32(area[1] - area[0])
    vd_s, vd_e = g("vortexEnforcingDomainStart"), g("vortexEnforcingDomainEnd")  # :54-57
    if vd_s is not None:
        p.has_vortex_domain = 1
        for d in range(dim):
            p.vd_start[d] = f32(vd_s[d])
            p.vd_end[d] = f32(vd_e[d])
    vscale = g("volumeScale")                                    # :17-19
    vp_volume = (float(vscale) if vscale is not None else 1.0) * m_V0
    p.vvpe_coef = f32(0.1592 * vp_volume)                        # :691
    p.eps = f32(1e-6)                                            # :15
    p.inv_eps = f32(1.0 / 1e-6)                                  # :16
    p.gen_a = f32(g("GenProbPara") if g("GenProbPara") is not None else 0.0)  # :58
    p.del_b = f32(g("DelProbPara") if g("DelProbPara") is not None else 0.0)  # :59
    p.kden_eps = f32(1e-8)                                       # :709
    p.kvn_eps = f32(1e-8)                                        # :316
    p.skip_cell0 = 1 if o.skip_cell0 else 0
    p.cell_origin_offset = 1 if o.cell_origin_offset else 0
    p.kernel_mode = DV_KERNEL_BLOB3D if o.kernel == "blob3d" else DV_KERNEL_REF2D
    delta = o.blob_delta if o.blob_delta is not None else r
    p.blob_delta2 = f32(delta * delta)
    p.blob_coef = f32(vp_volume / (4.0 * math.pi))
    p.compensated = 1 if o.compensated else 0
    if o.periodic:
        # cells of size box / floor(box / h) >= h, the same on every axis, so
        # the 3^d window around a cell holds every minimum-image neighbour
        n_cells = np.floor(domain_size / support).astype(int)
        gs = domain_size[0] / n_cells[0]
        for d in range(dim):
            if abs(domain_size[d] / n_cells[d] - gs) > 1e-9 * gs:
                raise ValueError("a periodic box needs the same cell size box/floor(box/h) on every axis")
            if n_cells[d] < 5:
                raise ValueError("a periodic box needs at least 5 cells per axis")
            p.grid_num[d] = int(n_cells[d])
            p.box[d] = f32(domain_size[d])
        p.grid_size = f32(gs)
        p.periodic = 1
        p.cell_origin_offset = 1
        p.skip_cell0 = 0
    return p


def derived(cfg) -> dict:
    """Host-side geometry that the reference keeps on ParticleSystem."""
    g = cfg.get_cfg
    domain_start = np.array(g("domainStart"), dtype=np.float64)
    domain_end = np.array(g("domainEnd"), dtype=np.float64)
    dim = len(domain_start)
    r = float(g("particleRadius"))
    support = r * 4.0
    return {
        "dim": dim,
        "domain_start": domain_start,
        "domain_end": domain_end,
        "domain_size": domain_end - domain_start,
        "particle_radius": r,
        "particle_diameter": 2 * r,
        "support_radius": support,
        "inv_support_radius": 1.0 / support,
        "m_V0": 0.8 * (2 * r) ** dim,
        "grid_num": np.ceil((domain_end - domain_start) / support).astype(int),
    }
