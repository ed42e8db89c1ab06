"""Differentiable vortex-particle rollout (periodic 2-D box): hand-written
adjoints against FP64 central differences, FP32 against FP64, the
differentiable forward against the production MC-VVPE, checkpoint recompute
against a stored tape, and the MC gradient against the full Biot-Savart
gradient."""
import numpy as np
import pytest
import torch

from dimcv_sph_b200 import scenes

pytestmark = pytest.mark.gpu

N = 16384      # 128 x 128 jittered lattice
EPS = 1e-6     # central-difference step (FP64)


def nrel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def vbox(cuda):
    from dimcv_sph_b200.adjoint import VortexBox
    cfg, x, w = scenes.periodic2d(N, seed=0, dt=0.01)
    box = VortexBox(cfg, x)
    w0 = torch.from_numpy(w).to(box.device)
    _, _, wt = scenes.periodic2d(N, seed=7, dt=0.01)
    return box, w0, torch.from_numpy(wt).to(box.device)


def _op_setup(box, w0):
    from dimcv_sph_b200.adjoint import MC
    w = w0.double()
    v = box.initial_velocity(w)
    plan = box.validate(box.build_plan(box.x0, v, 0, MC))
    plan.keep = True
    with torch.no_grad():
        box.velocity(box.x0.double(), w, plan)  # records the nominal positions
    return w, plan


def test_operator_gradient_matches_fp64_central_differences(vbox):
    box, w0, _ = vbox
    w, plan = _op_setup(box, w0)
    assert 0 < plan.n_src <= box.M and plan.nnz > 6 * box.n
    rng = np.random.default_rng(0)
    g = torch.from_numpy(rng.normal(size=(box.n, 2))).to(box.device)
    x = box.x0.double()
    xg = x.clone().requires_grad_(True)
    wg = w.clone().requires_grad_(True)
    L = (box.velocity(xg, wg, plan, frozen=True) * g).sum()
    gx, gw = torch.autograd.grad(L, (xg, wg))
    wc = rng.choice(box.n, 32, replace=False)
    xc = [(int(i), int(a)) for i, a in zip(rng.choice(box.n, 32, replace=False), rng.integers(0, 2, 32))]
    ad, fd = [], []
    with torch.no_grad():
        def f(xx, ww):
            return (box.velocity(xx, ww, plan, frozen=True) * g).sum().item()
        for c in wc:
            wp, wm = w.clone(), w.clone()
            wp[c] += EPS
            wm[c] -= EPS
            fd.append((f(x, wp) - f(x, wm)) / (2 * EPS))
            ad.append(gw[c].item())
        for i, a in xc:
            xp, xm = x.clone(), x.clone()
            xp[i, a] += EPS
            xm[i, a] -= EPS
            fd.append((f(xp, w) - f(xm, w)) / (2 * EPS))
            ad.append(gx[i, a].item())
    err = nrel(ad, fd)
    assert err < 1e-6, err
    # FP32 adjoint of the same plan against the FP64 one
    x32 = x.float().clone().requires_grad_(True)
    w32 = w.float().clone().requires_grad_(True)
    L32 = (box.velocity(x32, w32, plan) * g.float()).sum()
    gx32, gw32 = torch.autograd.grad(L32, (x32, w32))
    # FP32 sums of strongly cancelling far-field terms: ~1e-4 normwise
    assert nrel(gw32.cpu(), gw.cpu()) < 1e-3
    assert nrel(gx32.cpu(), gx.cpu()) < 1e-3


def test_differentiable_forward_matches_production_vvpe(vbox):
    """Smooth + Velocity (FP32) equals the library's MC-VVPE v_vort on the
    same samples when ω̃ is fed to it."""
    from dimcv_sph_b200.adjoint import MC
    box, w0, _ = vbox
    v = box.initial_velocity(w0)
    plan = box.validate(box.build_plan(box.x0, v, 0, MC))
    perm = plan.perm.long()
    with torch.no_grad():
        from dimcv_sph_b200.adjoint import _Smooth, _Velocity
        xs = box.x0.index_select(0, perm)
        ws = w0.index_select(0, perm)
        wt = _Smooth.apply(xs, ws, box, plan, None)
        us = _Velocity.apply(xs, wt, box, plan, None)
    sv = box.solver
    sv.d_vort_smoothed[: box.n] = 0
    sv.d_vort_smoothed[: box.n, 2] = wt
    sv.far_tile = 4
    sv.vort2vel()
    ref = sv.v_vort[: box.n, :2]
    assert torch.max(torch.abs(ref)) > 0
    assert nrel(us.cpu(), ref.cpu()) < 1e-5


def test_rollout_gradient_matches_fp64_central_differences(vbox):
    from dimcv_sph_b200.adjoint import VortexBox, fd_check
    box, w0, wt = vbox
    with torch.no_grad():
        target = box.rollout(wt.double(), 32)
    coords = np.random.default_rng(1).choice(box.n, 64, replace=False)
    ad, fd = fd_check(box, w0, target, coords, steps=32, eps=EPS)
    err = nrel(ad, fd)
    assert np.linalg.norm(fd) > 0
    assert err < 1e-5, err
    assert isinstance(VortexBox.loss(torch.zeros(2, 2), torch.ones(2, 2)).item(), float)


def test_checkpoint_recompute_is_bit_identical(vbox):
    box, w0, wt = vbox
    with torch.no_grad():
        target = box.rollout(wt, 16)
    grads = []
    for ck in (4, None):
        w = w0.clone().requires_grad_(True)
        L = box.loss(box.rollout(w, 16, checkpoint_every=ck), target)
        (g,) = torch.autograd.grad(L, w)
        grads.append(g)
    assert torch.equal(grads[0], grads[1])
    assert torch.count_nonzero(grads[0]) > box.n // 2


def test_mc_gradient_is_unbiased_for_full_biot_savart_gradient(vbox):
    """One MC gradient is a sparse, high-variance estimate of the full
    Biot-Savart gradient (only sampled particles carry far-field terms); the
    mean over independent sampler seeds converges to it like R^-1/2."""
    from dimcv_sph_b200.adjoint import FULL, MC
    box, w0, wt = vbox
    with torch.no_grad():
        target = box.rollout(wt, 32, mode=FULL)

    def grad(mode, seed=None):
        w = w0.clone().requires_grad_(True)
        L = box.loss(box.rollout(w, 32, mode=mode, seed=seed), target)
        return torch.autograd.grad(L, w)[0].double()

    ref = grad(FULL)
    gs = [grad(MC, 100 + r) for r in range(16)]
    e1 = np.mean([nrel(g.cpu(), ref.cpu()) for g in gs[:4]])
    e16 = nrel(torch.stack(gs).mean(0).cpu(), ref.cpu())
    mean16 = torch.stack(gs).mean(0)
    cos16 = float((mean16 * ref).sum() / (mean16.norm() * ref.norm()))
    assert e16 < e1 / 2.5, (e1, e16)
    assert cos16 > 0.6, cos16


def test_curl_matches_production_and_fp64_central_differences(vbox):
    """The SPH curl (ω from v) against the library's fused ∇v/ω sweep, and its
    VJP in x and v against FP64 central differences."""
    from dimcv_sph_b200.adjoint import MC
    box, w0, _ = vbox
    rng = np.random.default_rng(5)
    v = torch.from_numpy(rng.normal(0, 0.3, size=(box.n, 2)).astype(np.float32)).to(box.device)
    plan = box.validate(box.build_plan(box.x0, v, 0, MC))  # runs the production sweep on (x0, v)
    with torch.no_grad():
        w32 = box.curl(box.x0, v, plan)
    perm = plan.perm.long()
    prod = box.ps.vorticity[: box.n, 2]  # slot order
    assert nrel(w32.index_select(0, perm).cpu(), prod.cpu()) < 1e-5
    plan.keep = True
    x = box.x0.double()
    with torch.no_grad():
        box.velocity(x, w0.double(), plan)  # records the nominal positions
    vd = v.double()
    g = torch.from_numpy(rng.normal(size=box.n)).to(box.device)
    xg, vg = x.clone().requires_grad_(True), vd.clone().requires_grad_(True)
    L = (box.curl(xg, vg, plan, frozen=True) * g).sum()
    gx, gv = torch.autograd.grad(L, (xg, vg))

    def f(xx, vv):
        with torch.no_grad():
            return (box.curl(xx, vv, plan, frozen=True) * g).sum().item()

    ad, fd = [], []
    for _ in range(32):
        i, a = int(rng.integers(box.n)), int(rng.integers(2))
        vp, vm = vd.clone(), vd.clone()
        vp[i, a] += EPS
        vm[i, a] -= EPS
        fd.append((f(x, vp) - f(x, vm)) / (2 * EPS))
        ad.append(gv[i, a].item())
        xp, xm = x.clone(), x.clone()
        xp[i, a] += EPS
        xm[i, a] -= EPS
        fd.append((f(xp, vd) - f(xm, vd)) / (2 * EPS))
        ad.append(gx[i, a].item())
    assert nrel(ad, fd) < 1e-6, nrel(ad, fd)


def test_rollout_from_a_velocity_field(vbox):
    """ω0 = curl(x0, v0), then an 8-step rollout: the gradient in v0 (curl,
    smoothing and MC-VVPE adjoints chained) against FP64 central differences."""
    from dimcv_sph_b200.adjoint import MC
    box, w0, wt = vbox
    rng = np.random.default_rng(6)
    v0 = torch.from_numpy(rng.normal(0, 0.3, size=(box.n, 2))).to(box.device)
    with torch.no_grad():
        target = box.rollout(wt.double(), 8)
        _, plans = box.rollout(w0.double(), 8, mode=MC, keep_plans=True)
    for p in plans:
        box.validate(p)

    def loss(v, grad):
        with torch.set_grad_enabled(grad):
            w = box.curl(box.x0.double(), v, plans[0], frozen=True)
            return box.loss(box.rollout(w, 8, plans=plans, frozen=True, checkpoint_every=4), target)

    vg = v0.clone().requires_grad_(True)
    (g,) = torch.autograd.grad(loss(vg, True), vg)
    ad, fd = [], []
    for _ in range(24):
        i, a = int(rng.integers(box.n)), int(rng.integers(2))
        vp, vm = v0.clone(), v0.clone()
        vp[i, a] += EPS
        vm[i, a] -= EPS
        fd.append((loss(vp, False).item() - loss(vm, False).item()) / (2 * EPS))
        ad.append(g[i, a].item())
    assert np.linalg.norm(fd) > 0
    assert nrel(ad, fd) < 1e-5, nrel(ad, fd)
