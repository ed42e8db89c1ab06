"""dv_density_error_noalloc: the allocation-free density-error reduction.

Some callers cannot allocate device memory: real-time step loops that forbid
allocation once they run, and hosts whose own allocator owns all device
memory and hand this library only device pointers.  This entry point needs
no context and no cudaMalloc; its scratch is a fixed file-scope device array.
It still copies its result to the host and synchronises the stream, so it is
not used on a stream that is being captured.  The test calls it through the
C ABI twice in a row and checks both results against the context-based
dv_density_error on the same fields, within 1e-12 relative (both are FP64
sums of the same f32 terms in the same fixed order, so they agree exactly in
practice).  The scenes cover 2-D with and without the divergence transit
weight and the 3-D sphere scene; an empty range must give exactly 0.

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

SCENES = {
    "channel2d_transit": lambda: scenes.channel2d(length=2.0, reserved=200, transit=True),
    "channel2d_plain": lambda: scenes.channel2d(length=2.0, reserved=200, transit=False),
    "sphere3d_coarse": lambda: scenes.sphere3d(radius=0.016, dt=6.4e-4),
}


def _scene(name="channel2d_transit"):
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(SCENES[name]())
    solver = ps.build_solver()
    n = ps.particle_num[None]
    # a seeded velocity disturbance so that the density change is not zero
    rng = np.random.default_rng(1)
    fl = ps.material[:n] == 1
    noise = torch.from_numpy(rng.normal(0, 0.3, size=(n, ps.dim)).astype(np.float32)).to(ps.device)
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


@pytest.mark.parametrize("name", list(SCENES))
def test_noalloc_matches_context_entry_point_twice(cuda, name):
    ps, solver = _scene(name)
    assert bool(ps.params.has_transit) == (name == "channel2d_transit")
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


def test_noalloc_empty_range_is_zero(cuda):
    ps, solver = _scene()
    solver.compute_density_change()
    assert _noalloc(ps, ps.particle_num[None], 0.0) != 0.0  # leaves non-zero partials behind
    for _ in range(2):
        assert _noalloc(ps, 0, 0.0) == 0.0


def test_noalloc_rejects_sizes_beyond_the_limit(cuda):
    ps, _ = _scene()
    out = C.c_double(0.0)
    rc = ps.lib.dv_density_error_noalloc(C.byref(ps.params), C.byref(ps.fields_struct), (1 << 24) + 1,
                                         0.0, C.byref(out), C.c_void_p(ps.stream.cuda_stream))
    assert rc == _abi.DV_ECAPACITY
    assert b"16777216" in ps.lib.dv_last_error(None)
