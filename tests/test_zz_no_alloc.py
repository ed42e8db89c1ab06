"""dv_density_error_noalloc: the allocation-free density-error reduction.

Some callers cannot allocate device memory: a stream captured in the global
capture mode (cudaMalloc fails there), real-time step loops that forbid
allocation after start-up, or hosts whose allocator owns all device memory.
This entry point needs no context and no cudaMalloc; its scratch is a fixed
file-scope device array.  The test calls it through the C ABI twice in a row
and checks both results against the context-based dv_density_error on the
same fields, within 1e-12 relative (both are FP64 sums of the same f32 terms
in the same fixed order, so they agree exactly in practice).

This file sorts last on purpose: a failure here stops a `-x` run only after
every other test has run.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from dimcv_sph_b200 import _abi, scenes

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _scene():
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(scenes.channel2d(length=2.0, reserved=200))
    solver = ps.build_solver()
    n = ps.particle_num[None]
    # a seeded velocity disturbance so that the density change is not zero
    rng = np.random.default_rng(1)
    fl = ps.material[:n] == 1
    noise = torch.from_numpy(rng.normal(0, 0.3, size=(n, 2)).astype(np.float32)).to(ps.device)
    ps.v[:n] += torch.where(fl.unsqueeze(1), noise, torch.zeros_like(noise))
    solver.initialize()
    solver.compute_densities()
    solver.compute_DFSPH_factor()
    return ps, solver


def _noalloc(ps, n, offset):
    out = C.c_double(float("nan"))
    rc = ps.lib.dv_density_error_noalloc(C.byref(ps.params), C.byref(ps.fields_struct), n,
                                         float(np.float32(offset)), C.byref(out),
                                         C.c_void_p(ps.stream.cuda_stream))
    assert rc == 0, ps.lib.dv_last_error(None)
    return out.value


def test_noalloc_matches_context_entry_point_twice(cuda):
    ps, solver = _scene()
    n = ps.particle_num[None]
    solver.compute_density_change()
    ref0 = solver.compute_density_error(0.0)
    assert ref0 != 0.0
    solver.compute_density_adv()
    ref1 = solver.compute_density_error(solver.density_0)
    assert ref1 != 0.0
    for _ in range(2):  # consecutive calls share the scratch array
        got1 = _noalloc(ps, n, solver.density_0)
        assert abs(got1 - ref1) <= RTOL * abs(ref1)
    solver.compute_density_change()
    for _ in range(2):
        got0 = _noalloc(ps, n, 0.0)
        assert abs(got0 - ref0) <= RTOL * abs(ref0)


def test_noalloc_rejects_sizes_beyond_the_limit(cuda):
    ps, _ = _scene()
    out = C.c_double(0.0)
    rc = ps.lib.dv_density_error_noalloc(C.byref(ps.params), C.byref(ps.fields_struct), (1 << 24) + 1,
                                         0.0, C.byref(out), C.c_void_p(ps.stream.cuda_stream))
    assert rc == _abi.DV_ECAPACITY
    assert b"16777216" in ps.lib.dv_last_error(None)
