"""The Monte-Carlo error of the inverse-CDF sampler against the reference's
own estimator.

The reference draws its samples by a Bernoulli birth/death process on the
kinematic vorticity number (``dimcv_sph.py:305-335``) and weights each far
sample by ``(kden_sum - S_i) / (kden_s + 1e-8)`` (``:696-714``); the number of
samples is whatever the process gives.  This build adds inverse-CDF draws of
M samples from p ∝ kden.  Both estimators are run on identical states, the
inverse-CDF one with M equal to the Bernoulli count of that state, for 16
seeds each, and both v_vort fields (before the gate) are compared with the
FP64 full Biot-Savart sum of the same kernel (the near plus far sum the
estimator approximates, ``dv_bs_full`` precision 64):

* the 2-D channel (r = 0.01, about 10k fluid) after 50 steps of flow under
  the Bernoulli sampler, so that the sample set has its natural history;
* the 3-D vortex ring (32,768 particles, the reference's 2-D projected
  kernel), one birth/death draw from an empty sample set.

The test asserts that the mean inverse-CDF error is at most the upper end of
the 95% confidence interval of the mean Bernoulli error (t quantile, 15
degrees of freedom), and prints both distributions.
"""
import ctypes as C
import json

import numpy as np
import pytest
import torch

from dimcv_sph_b200 import _lib, scenes
from dimcv_sph_b200._abi import DV_SAMPLE_INVERSE_CDF

pytestmark = pytest.mark.gpu

SEEDS = 16
T975_15 = 2.131  # Student t, 97.5% quantile, 15 degrees of freedom


def _bs64(ps, omega, n):
    out = torch.zeros((n, 4), dtype=torch.float64, device=ps.device)
    rc = ps.lib.dv_bs_full(ps.ctx, C.byref(ps.fields_struct), C.c_void_p(omega.data_ptr()), None, n,
                           C.c_void_p(out.data_ptr()), 64)
    _lib.check(ps.ctx, rc, "dv_bs_full")
    return out[:, :3]


def _rel_rms(est, ref, rows):
    e = (est[rows].double() - ref[rows]) ** 2
    return float(torch.sqrt(e.sum(1).mean()) / torch.sqrt((ref[rows] ** 2).sum(1).mean()))


def _verdict(name, eb, ei, mb):
    eb, ei = np.array(eb), np.array(ei)
    upper = eb.mean() + T975_15 * eb.std(ddof=1) / np.sqrt(len(eb))
    print(json.dumps({"case": name, "mean_bernoulli_samples": float(np.mean(mb)),
                      "bernoulli": {"mean": eb.mean(), "std": eb.std(ddof=1), "upper95": upper,
                                    "all": eb.round(5).tolist()},
                      "inverse_cdf": {"mean": ei.mean(), "std": ei.std(ddof=1), "all": ei.round(5).tolist()}}))
    assert ei.mean() <= upper, (name, ei.mean(), upper)


def test_channel_after_50_steps(cuda):
    from dimcv_sph_b200.particle_system import ParticleSystem
    eb, ei, mb = [], [], []
    for seed in range(SEEDS):
        ps = ParticleSystem(scenes.channel2d(sampler="bernoulli", seed=seed))
        s = ps.build_solver()
        s.initialize()
        for _ in range(50):
            s.step()
        # the substep of step 51 up to the VVPE, Bernoulli samples
        if s.cnt % s.emit_interval == 0:
            s.emit_particle()
        s.cnt += 1
        ps.initialize_particle_system()
        s.compute_densities()
        s.compute_DFSPH_factor()
        s.divergence_solve()
        s.compute_non_pressure_forces()
        s.init()
        s.compute_d_vorticity()
        s.compute_all_d_vort_smoothed()
        s.update_sample()
        s.compute_kernel_density()
        n = ps.particle_num[None]
        M = ps.counters()["num_samples"]
        assert M > 0
        s.vort2vel()
        v_b = s.v_vort[:n].clone()
        # inverse-CDF draws of the same count on the same state
        s._calls("dv_sample", DV_SAMPLE_INVERSE_CDF, seed, 10_000 + seed, M)
        s.vort2vel()
        v_i = s.v_vort[:n].clone()
        ref = _bs64(ps, ps.solver_buf.t["d_vort_smoothed"], n)
        fl = ps.material[:n] == 1
        eb.append(_rel_rms(v_b, ref, fl))
        ei.append(_rel_rms(v_i, ref, fl))
        mb.append(M)
        del s, ps
    _verdict("channel2d after 50 steps", eb, ei, mb)


def test_ring_reference_kernel(cuda):
    from dimcv_sph_b200.ring_study import RingStudy
    st = RingStudy(n=32768, subset=4096, kernel3d=False)
    ps, s = st.ps, st.solver
    eb, ei, mb = [], [], []
    for seed in range(SEEDS):
        ps.v[: st.n] = st.v0
        ps.initialize_particle_system()
        s.init()
        ps.is_sample[: ps.particle_num[None]] = 0
        s._calls("dv_kvn_sample", seed, 0, 1)  # one birth/death draw (dimcv_sph.py:305-324)
        s._calls("dv_record_samples")
        s.compute_kernel_density()
        M = ps.counters()["num_samples"]
        assert M > 0
        s.vort2vel()
        eb.append(st.mc_error())
        s._calls("dv_sample", DV_SAMPLE_INVERSE_CDF, seed, 20_000 + seed, M)
        s.vort2vel()
        ei.append(st.mc_error())
        mb.append(M)
    _verdict("ring3d, reference kernel", eb, ei, mb)
