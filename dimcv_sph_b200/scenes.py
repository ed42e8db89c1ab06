"""Scene builders for the benchmark and test configurations.

All inputs are synthetic and seeded; they use the reference's scene-JSON
schema (data/scenes/von_karman_vortex_street.json) plus the new keys this
build understands (samplerMode, mcSamples, seed, cylinderCenter/Radius,
obstacleShape, kernel3D, cellOriginOffset, skipCell0, exclude/keepInside).

  channel2d  2-D von Kármán channel [0,4]×[0,1], r = 0.01 (~9k fluid + ~0.9k
             boundary), inflow 1 m/s, cylinder r = 0.1 at (1.0, 0.5),
             dt = 4e-4, M = N/16 inverse-CDF samples, seed 0.
  sphere3d   flow past a sphere (r = 0.15) in a 3×1×1 box, r = 0.004
             (~2.0M fluid + ~0.3M boundary), inflow 1 m/s, M = N/32.
  ring3d     operator-level: N points uniform in [-1,1]³ with a Gaussian-core
             vortex ring (R 0.5, σ 0.05, Γ 1) plus N(0, 1e-3) noise.
"""
from __future__ import annotations

import math

import numpy as np

from .config_builder import SimConfig

_FLUID_COLOR = [50, 100, 200]
_SOLID_COLOR = [201, 112, 100]


def _block(obj, start, end, velocity, **extra):
    d = {"objectId": obj, "start": list(start), "end": list(end), "translation": [0.0] * len(start),
         "scale": [1] * len(start), "velocity": list(velocity), "density": 1000.0}
    d.update(extra)
    return d


def channel2d(radius=0.01, length=4.0, height=1.0, inflow=1.0, cyl_center=(1.0, 0.5), cyl_radius=0.1,
              dt=4e-4, mc_fraction=1.0 / 16.0, sampler="inverse_cdf", seed=0, reserved=4000,
              transit=True, trim_cylinder=False) -> SimConfig:
    """trim_cylinder=True builds the obstacle the reference way: a solid
    square that init_cylinder trims, moving the trimmed particles to the
    origin (karman_vortex.py:27-36)."""
    d = 2 * radius
    wall = 2 * d  # two particle layers
    cfg = {
        "Configuration": {
            "domainStart": [0.0, 0.0], "domainEnd": [length, height],
            "particleRadius": radius, "numberOfStepsPerRenderUpdate": 1, "density0": 1000,
            "simulationMethod": 0, "gravitation": [0.0, 0.0], "timeStepSize": dt,
            "bounceBackBoundary": False, "simulationTime": 200 * dt,
            "volumeScale": 0.2, "GenProbPara": 5, "DelProbPara": 3.5,
            "reservedCapacity": reserved, "exportPLY": False,
            "cylinderCenter": [cyl_center[0], cyl_center[1], 0.5], "cylinderRadius": cyl_radius,
            "samplerMode": sampler, "mcSamples": mc_fraction, "seed": seed,
        },
        "FluidEmitters": [{
            "objectId": 0, "squareCenter": [0.0, height / 2], "squareSize": [0.0, height - 2 * wall],
            "velocity": [inflow, 0.0], "density": 1000.0, "color": _FLUID_COLOR}],
        "FluidBlocks": [_block(3, [d, wall], [length, height - wall], [inflow, 0.0], color=_FLUID_COLOR,
                               exclude=[{"center": list(cyl_center), "radius": cyl_radius + 0.5 * d}])],
        "RigidBlocks": [
            _block(1, [0.0, 0.0], [length, wall], [0.0, 0.0], color=_SOLID_COLOR, isDynamic=False),
            _block(1, [0.0, height - wall], [length, height], [0.0, 0.0], color=_SOLID_COLOR, isDynamic=False),
            _block(2, [cyl_center[0] - cyl_radius, cyl_center[1] - cyl_radius],
                   [cyl_center[0] + cyl_radius + 1e-9, cyl_center[1] + cyl_radius + 1e-9], [0.0, 0.0],
                   color=_SOLID_COLOR, isDynamic=False,
                   keepInside={"center": list(cyl_center), "radius": cyl_radius}),
        ],
    }
    if transit:
        cfg["Configuration"]["divergenceTransitArea"] = [0.0, 0.02]
    if trim_cylinder:
        del cfg["RigidBlocks"][2]["keepInside"]
    return SimConfig(config=cfg)


def sphere3d(radius=0.004, size=(3.0, 1.0, 1.0), inflow=1.0, center=(0.5, 0.5, 0.5), sphere_radius=0.15,
             fluid_length=1.1, dt=1.6e-4, mc_fraction=1.0 / 32.0, sampler="inverse_cdf", seed=0,
             reserved=None) -> SimConfig:
    d = 2 * radius
    wall = 2 * d
    L, H, W = size
    cfg = {
        "Configuration": {
            "domainStart": [0.0, 0.0, 0.0], "domainEnd": [L, H, W],
            "particleRadius": radius, "numberOfStepsPerRenderUpdate": 1, "density0": 1000,
            "simulationMethod": 0, "gravitation": [0.0, 0.0, 0.0], "timeStepSize": dt,
            "bounceBackBoundary": False, "simulationTime": 100 * dt,
            "volumeScale": 0.2, "GenProbPara": 5, "DelProbPara": 3.5, "exportPLY": False,
            "cylinderCenter": list(center), "cylinderRadius": sphere_radius, "obstacleShape": "sphere",
            "samplerMode": sampler, "mcSamples": mc_fraction, "seed": seed,
        },
        "FluidEmitters": [{
            "objectId": 0, "squareCenter": [0.0, H / 2, (wall + W) / 2],
            "squareSize": [0.0, H - 2 * wall, W - wall], "velocity": [inflow, 0.0, 0.0],
            "density": 1000.0, "color": _FLUID_COLOR}],
        "FluidBlocks": [_block(3, [d, wall, wall], [fluid_length, H - wall, W], [inflow, 0.0, 0.0],
                               color=_FLUID_COLOR,
                               exclude=[{"center": list(center), "radius": sphere_radius + 0.5 * d}])],
        "RigidBlocks": [
            _block(1, [0.0, 0.0, 0.0], [L, wall, W], [0.0] * 3, color=_SOLID_COLOR, isDynamic=False),
            _block(1, [0.0, H - wall, 0.0], [L, H, W], [0.0] * 3, color=_SOLID_COLOR, isDynamic=False),
            _block(1, [0.0, wall, 0.0], [L, H - wall, wall], [0.0] * 3, color=_SOLID_COLOR, isDynamic=False),
            _block(2, [c - sphere_radius for c in center], [c + sphere_radius + 1e-9 for c in center],
                   [0.0] * 3, color=_SOLID_COLOR, isDynamic=False,
                   keepInside={"center": list(center), "radius": sphere_radius}),
        ],
    }
    if reserved is not None:
        cfg["Configuration"]["reservedCapacity"] = reserved
    else:
        # room for the emissions of 100 steps
        per = int(math.ceil((H - 2 * wall) / d)) * int(math.ceil((W - wall) / d))
        steps_per_emit = int(math.ceil(d / (inflow * np.float32(dt))))
        cfg["Configuration"]["reservedCapacity"] = per * (100 // steps_per_emit + 2)
    return SimConfig(config=cfg)


def periodic_blobs(x: np.ndarray, seed: int, n_blobs=8) -> np.ndarray:
    """Vorticity (z) of n_blobs Gaussian blobs on the unit periodic square:
    amplitude N(0, 5), width σ ~ U(0.03, 0.08), centres uniform; distances
    by minimum image."""
    rng = np.random.default_rng(seed)
    centers = rng.uniform(0.0, 1.0, size=(n_blobs, 2))
    amps = rng.normal(0.0, 5.0, size=n_blobs)
    sig = rng.uniform(0.03, 0.08, size=n_blobs)
    w = np.zeros(x.shape[0])
    for c, a, s in zip(centers, amps, sig):
        d = x[:, :2] - c
        d -= np.round(d)
        w += a * np.exp(-(d * d).sum(1) / (s * s))
    return w


def periodic2d(n: int = 65536, seed: int = 0, jitter: float = 0.25, dt: float = 1e-3):
    """(config, positions float32 [n,2], vorticity float32 [n]) on the unit
    periodic square: a jittered √n × √n lattice (jitter U(-j, j)·spacing),
    particle radius = spacing / 2 (h = 2 spacings), volume 1/n per particle."""
    k = int(round(math.sqrt(n)))
    if k * k != n:
        raise ValueError("n must be a square number")
    sp = 1.0 / k
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(k), np.arange(k), indexing="ij"), -1).reshape(-1, 2)
    x = (g + 0.5) * sp + rng.uniform(-jitter, jitter, size=g.shape) * sp
    x = np.mod(x, 1.0)
    w = periodic_blobs(x, seed + 1)
    cfg = {
        "Configuration": {
            "domainStart": [0.0, 0.0], "domainEnd": [1.0, 1.0], "particleRadius": sp / 2,
            "density0": 1000, "simulationMethod": 0, "gravitation": [0.0, 0.0], "timeStepSize": dt,
            # vp_volume = volumeScale * 0.8 (2r)^2 = 1/n
            "volumeScale": 1.25, "GenProbPara": 5, "DelProbPara": 3.5, "periodic": True,
            "samplerMode": "stratified", "seed": seed,
        },
    }
    x32 = x.astype(np.float32)
    x32[x32 >= np.float32(1.0)] = 0.0  # 1 - tiny rounds to 1 in f32: the same point as 0
    return SimConfig(config=cfg), x32, w.astype(np.float32)


def ring_vorticity(x: np.ndarray, R=0.5, sigma=0.05, gamma=1.0) -> np.ndarray:
    """Gaussian-core vortex ring in the x-y plane about the z axis:
    ω = Γ/(πσ²) exp(-d²/σ²) e_θ with d the distance to the core circle."""
    rho = np.sqrt(x[:, 0] ** 2 + x[:, 1] ** 2)
    d2 = (rho - R) ** 2 + x[:, 2] ** 2
    mag = gamma / (math.pi * sigma * sigma) * np.exp(-d2 / (sigma * sigma))
    rs = np.maximum(rho, 1e-12)
    w = np.zeros_like(x)
    w[:, 0] = -x[:, 1] / rs * mag
    w[:, 1] = x[:, 0] / rs * mag
    return w


def ring3d(n: int = 1 << 20, seed: int = 0, noise=1e-3, kernel3d=True):
    """(config, positions float32 [n,3], vorticity float32 [n,3]).  Particle
    radius r = ½(8/n)^{1/3} (h = 4r), volume per particle V = 8/n."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, size=(n, 3))
    w = ring_vorticity(x) + rng.normal(0.0, noise, size=(n, 3))
    r = 0.5 * (8.0 / n) ** (1.0 / 3.0)
    cfg = {
        "Configuration": {
            "domainStart": [-1.0, -1.0, -1.0], "domainEnd": [1.0, 1.0, 1.0],
            "particleRadius": r, "density0": 1000, "simulationMethod": 0,
            "gravitation": [0.0, 0.0, 0.0], "timeStepSize": 1e-3,
            # vp_volume = volumeScale * 0.8 (2r)^3 = 8/n
            "volumeScale": 1.25, "GenProbPara": 5, "DelProbPara": 3.5,
            "cellOriginOffset": True, "skipCell0": False, "kernel3D": bool(kernel3d),
            "blobDelta": r, "samplerMode": "inverse_cdf", "seed": seed,
        },
    }
    return SimConfig(config=cfg), x.astype(np.float32), w.astype(np.float32)
