"""Statistical checks of the Monte-Carlo VVPE on the GPU (vortex ring,
blob kernel) against the FP64 full Biot-Savart sum, and of the FP64-CDF
inverse-CDF sampler against its target distribution p ∝ kden."""
import ctypes as C

import numpy as np
import pytest
import torch

from dimcv_sph_b200._abi import DV_SAMPLE_INVERSE_CDF

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ring(cuda):
    from dimcv_sph_b200.ring_study import RingStudy
    return RingStudy(n=32768, subset=4096)


def test_full_bs_fp32_accuracy(ring):
    errs = {}
    for comp in (False, True):
        ring.set_compensated(comp)
        u = ring.bs(ring.sub, ring.sub.numel(), 32)[:, :3].double()
        errs[comp] = float(torch.sqrt(((u - ring.uref) ** 2).sum(1).mean())) / ring.uref_rms
    ring.set_compensated(False)
    assert errs[False] < 1e-5 and errs[True] < 1e-5
    assert errs[True] <= errs[False] * 1.5


def test_mc_error_falls_with_M(ring):
    res = {}
    for M in (512, 2048, 8192):
        e = []
        for k in range(4):
            ring.mc_step(M, 100 + k)
            e.append(ring.mc_error())
        res[M] = float(np.mean(e))
    # RMS error ∝ M^-1/2: a 16x larger M should cut it by ~4 (accept 2.5)
    assert res[8192] < res[2048] < res[512]
    assert res[512] / res[8192] > 2.5, res


def test_mc_mean_is_unbiased(ring):
    """Mean of K independent estimates vs the FP64 sum: the bias must sit
    within 3 standard errors of the mean (per-target, aggregated RMS)."""
    K, M = 16, 1024
    est = []
    for k in range(K):
        ring.mc_step(M, 500 + k)
        est.append(ring.solver.v_vort[ring.sub.long()].double().clone())
    est = torch.stack(est)  # K x S x 3
    mean = est.mean(0)
    se = est.std(0) / np.sqrt(K)
    bias = (mean - ring.uref).abs()
    frac_outside = float(((bias > 3 * se + 1e-7 * ring.uref_rms)).double().mean())
    assert frac_outside < 0.02, frac_outside


def test_inverse_cdf_draws_follow_kden(ring):
    ps, s = ring.ps, ring.solver
    n = ring.n
    ring.mc_step(64, 1)  # computes kden for this state
    M = n  # the sample buffer holds at most `capacity` draws
    s._calls("dv_sample", DV_SAMPLE_INVERSE_CDF, 3, 9, M)
    idx = s.sample_idx[:M].long()
    counts = torch.bincount(idx, minlength=n).double().cpu().numpy()
    kden = s.kernel_density[:n].double().cpu().numpy()
    p = kden / kden.sum()
    # chi-square over 32 equal-probability groups of slots (ordered by kden)
    order = np.argsort(p)
    cp = np.cumsum(p[order])
    groups = np.minimum((cp * 32).astype(int), 31)
    obs = np.bincount(groups, weights=counts[order], minlength=32)
    exp = np.bincount(groups, weights=p[order], minlength=32) * M
    keep = exp > 5
    chi2 = float(((obs[keep] - exp[keep]) ** 2 / exp[keep]).sum())
    dof = int(keep.sum()) - 1
    # p-value > 1e-4  <=>  chi2 below ~ dof + 8 sqrt(2 dof) for these dof
    assert chi2 < dof + 8 * np.sqrt(2 * dof), (chi2, dof)
    assert counts[kden == 0].sum() == 0
