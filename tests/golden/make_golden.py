"""Generates the golden fixtures that pin the C++ oracle.

A second, independent restatement of the reference (Haok-Z/DIMCV-SPH) in
NumPy f32: neighbours by brute force over all pairs (|x_i - x_j| < h in f32,
the 3^d-cell window of particle_system.py:562-586 and its flat-cell-0 quirk),
then the substep kernels of dimcv_sph.py / sph_base.py evaluated per particle.
It shares no code with the oracle or the CUDA library; it only imports the
parameter derivation (dimcv_sph_b200.params), whose constants it checks
itself.  The reference cannot be run here (Taichi is not installed), so these
fixtures pin the oracle to a restatement, not to reference output.

Run:  python tests/golden/make_golden.py   (writes tests/golden/*.npz)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from dimcv_sph_b200.config_builder import SimConfig  # noqa: E402
from dimcv_sph_b200.params import make_params  # noqa: E402

F = np.float32


def scene(dim: int, seed: int):
    """Small jittered lattice of fluid over a two-layer solid floor."""
    rng = np.random.default_rng(seed)
    r = 0.01
    d = 2 * r
    if dim == 2:
        nx, ny = 12, 9
        g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij"), -1).reshape(-1, 2)
        fluid = (g + [1, 3]) * d + rng.uniform(-0.2, 0.2, size=g.shape) * d
        fl = np.stack(np.meshgrid(np.arange(nx + 2), np.arange(2), indexing="ij"), -1).reshape(-1, 2)
        solid = (fl + [0, 0.5]) * d
        dom = [0.0, 0.0], [0.4, 0.3]
    else:
        nx = 6
        g = np.stack(np.meshgrid(*[np.arange(nx)] * 3, indexing="ij"), -1).reshape(-1, 3)
        fluid = (g + [1, 1, 3]) * d + rng.uniform(-0.2, 0.2, size=g.shape) * d
        fl = np.stack(np.meshgrid(np.arange(nx + 2), np.arange(nx + 2), np.arange(2), indexing="ij"),
                      -1).reshape(-1, 3)
        solid = (fl + [0, 0, 0.5]) * d
        dom = [0.0, 0.0, 0.0], [0.2, 0.2, 0.2]
    x = np.concatenate([fluid, solid]).astype(F)
    nf = fluid.shape[0]
    mat = np.concatenate([np.ones(nf, np.int32), np.zeros(solid.shape[0], np.int32)])
    v = np.zeros_like(x)
    v[:nf] = rng.normal(0, 0.3, size=(nf, dim)).astype(F)
    cfg = SimConfig(config={"Configuration": {
        "domainStart": dom[0], "domainEnd": dom[1], "particleRadius": r, "density0": 1000,
        "timeStepSize": 4e-4, "gravitation": [0.0] * (dim - 1) + [-9.81], "volumeScale": 0.2,
        "GenProbPara": 5, "DelProbPara": 3.5}})
    return cfg, x, v, mat


def run(dim: int, seed: int) -> dict:
    cfg, x, v, mat = scene(dim, seed)
    P = make_params(cfg)
    n = x.shape[0]
    h = F(P.support_radius)
    inv_h = F(P.inv_support_radius)
    # constants checked independently of params.py
    k_dim = F({2: 1.8189, 3: 2.5465}[dim])
    hd = F(inv_h * inv_h) if dim == 2 else F(F(inv_h * inv_h) * inv_h)
    assert F(P.kW) == F(k_dim * hd)
    assert F(P.kG) == F(F(F(6.0) * k_dim) * hd)

    cell = (x / F(P.grid_size)).astype(np.int32)
    gn = np.array(P.grid_num[:dim])
    mV0 = F(0.8 * (2 * 0.01) ** dim)
    mV = np.full(n, mV0, F)
    m = (mV * F(1000.0)).astype(F)
    rng = np.random.default_rng(seed + 100)

    def W(rn):
        q = F(rn * inv_h)
        if q <= 1.0:
            if q <= 0.5:
                q2 = F(q * q)
                q3 = F(q2 * q)
                return F(F(P.kW) * F(F(F(F(6.0) * q3) - F(F(6.0) * q2)) + F(1.0)))
            f = F(F(1.0) - q)
            return F(F(P.kW2) * F(F(f * f) * f))
        return F(0.0)

    def gradW(r):
        rn = F(np.sqrt(sqn(r)))
        q = F(rn * inv_h)
        res = np.zeros(dim, F)
        if rn > F(1e-5) and q <= 1.0:
            gq = np.array([F(F(r[c] / rn) * inv_h) for c in range(dim)], F)
            if q <= 0.5:
                s = F(F(F(P.kG) * q) * F(F(F(3.0) * q) - F(2.0)))
            else:
                f = F(F(1.0) - q)
                s = F(F(P.kG) * F(-F(f * f)))
            res = np.array([F(s * gq[c]) for c in range(dim)], F)
        return res

    def sqn(r):
        s = F(F(r[0] * r[0]) + F(r[1] * r[1]))
        if dim == 3:
            s = F(s + F(r[2] * r[2]))
        return s

    # brute-force neighbour sets with the cell window and the cell-0 rule
    nbrs = []
    for i in range(n):
        lst = []
        for j in range(n):
            if j == i:
                continue
            if np.any(np.abs(cell[j] - cell[i]) > 1) or np.any(cell[j] < 0) or np.any(cell[j] >= gn):
                continue
            if np.all(cell[j] == 0):
                continue
            r = (x[i] - x[j]).astype(F)
            if F(np.sqrt(sqn(r))) < h:
                lst.append(j)
        nbrs.append(lst)

    fluid = mat == 1
    density = np.zeros(n, F)
    factor = np.zeros(n, F)
    dchange = np.zeros(n, F)
    acc = np.zeros((n, dim), F)
    vort = np.zeros((n, 3), F)
    gradv = np.zeros((n, dim, dim), F)
    kvn = np.zeros(n, F)
    kden = np.zeros(n, F)
    g = np.array([0.0] * (dim - 1) + [-9.81], F)
    for i in range(n):
        if not fluid[i]:
            continue
        den = F(0.0)
        gi = np.zeros(dim, F)
        sk = F(0.0)
        adv = F(0.0)
        a = g.copy()
        w3 = np.zeros(3, F)
        gv = np.zeros((dim, dim), F)
        for j in nbrs[i]:
            r = (x[i] - x[j]).astype(F)
            rn = F(np.sqrt(sqn(r)))
            den = F(den + F(mV[j] * W(rn)))
            gw = gradW(r)
            dv = (v[i] - v[j]).astype(F)
            dot = F(F(dv[0] * gw[0]) + F(dv[1] * gw[1]))
            if dim == 3:
                dot = F(dot + F(dv[2] * gw[2]))
            adv = F(adv + F(mV[j] * dot))
            if fluid[j]:
                gp = (m[j] * gw).astype(F)
                sk = F(sk + sqn(gp))
                gi = (gi + gp).astype(F)
                vxy = F(F(dv[0] * r[0]) + F(dv[1] * r[1]))
                if dim == 3:
                    vxy = F(vxy + F(dv[2] * r[2]))
                s = F(F(F(F(P.visc_coef) * mV[j]) * vxy) / F(F(rn * rn) + F(P.visc_h2)))
                a = (a + (s * gw).astype(F)).astype(F)
                vji = np.zeros(3, F)
                vji[:dim] = (v[j] - v[i]).astype(F)
                g3 = np.zeros(3, F)
                g3[:dim] = gw
                cr = np.array([F(F(vji[1] * g3[2]) - F(vji[2] * g3[1])),
                               F(F(vji[2] * g3[0]) - F(vji[0] * g3[2])),
                               F(F(vji[0] * g3[1]) - F(vji[1] * g3[0]))], F)
                w3 = (w3 + (mV[j] * cr).astype(F)).astype(F)
                for p in range(dim):
                    for q in range(dim):
                        gv[p, q] = F(gv[p, q] + F(F(mV[j] * vji[p]) * gw[q]))
            else:
                sm = F(mV[j] * F(1000.0))
                gi = (gi + (sm * gw).astype(F)).astype(F)
        density[i] = F(F(F(mV[i] * W(F(0.0))) + den) * F(1000.0))
        sk = F(sk + sqn(gi))
        factor[i] = F(F(1.0) / sk) if sk > F(1e-6) else F(0.0)
        da = max(adv, F(0.0))
        dchange[i] = F(0.0) if len(nbrs[i]) < P.neighbor_min else da
        acc[i] = a
        vort[i] = w3
        gradv[i] = gv
        Wt = (gv - gv.T).astype(F)
        St = (gv + gv.T).astype(F)
        kvn[i] = F(F(np.sqrt(F(np.sum((Wt * Wt).astype(np.float64)))))
                   / F(F(np.sqrt(F(np.sum((St * St).astype(np.float64))))) + F(1e-8)))
    # AKDE (Epanechnikov, dimcv_sph.py:721-751)
    def epan(r):
        ret = F(1.0)
        for c in range(dim):
            q = F(abs(r[c]) * inv_h)
            ret = F(ret * F(F(0.75) * F(F(1.0) - F(q * q)))) if q < 1.0 else F(0.0)
        return ret
    for i in range(n):
        if not fluid[i]:
            continue
        kd = F(kvn[i] * epan(np.zeros(dim, F)))
        for j in nbrs[i]:
            if fluid[j]:
                kd = F(kd + F(kvn[j] * epan((x[i] - x[j]).astype(F))))
        kden[i] = kd
    # VVPE with injected samples (dimcv_sph.py:649-719), ω̃ set to a random field
    wt = np.zeros((n, 3), F)
    wt[fluid, 2 if dim == 2 else slice(0, 3)] = rng.normal(0, 1.0, size=(fluid.sum(),) if dim == 2
                                                           else (fluid.sum(), 3)).astype(F)
    samples = np.sort(rng.choice(np.nonzero(fluid)[0], size=max(4, fluid.sum() // 8), replace=False))
    kden_sum = F(np.sum(kden[fluid].astype(np.float64)))
    vv = np.zeros((n, 3), np.float64)
    coef = np.float64(F(P.vvpe_coef))
    for i in np.nonzero(fluid)[0]:
        near = np.zeros(3)
        S = np.float64(kden[i])
        for j in nbrs[i]:
            if not fluid[j]:
                continue
            r = (x[i] - x[j]).astype(np.float64)
            rp = np.array([r[0], r[1], 0.0])
            rn = np.sqrt(rp[0] ** 2 + rp[1] ** 2)
            K = (1 - np.exp(-rn * 1e6)) / (rn * (rn + 1e-6 * np.exp(-rn * 1e6)))
            near += K * np.cross(rp, wt[j].astype(np.float64))
            S += kden[j]
        far = np.zeros(3)
        cnt = 0
        for j in samples:
            r32 = (x[i] - x[j]).astype(F)
            if not F(np.sqrt(sqn(r32))) > h:
                continue
            r = r32.astype(np.float64)
            rn = np.sqrt(np.sum(r * r))
            rp = np.array([r[0], r[1], 0.0])
            far += (1.0 / (rn * rn)) * np.cross(rp, wt[j]) * (np.float64(kden_sum) - S) / (np.float64(kden[j]) + 1e-8)
            cnt += 1
        vv[i] = near * coef + (far * coef / cnt if cnt else 0.0)
    off = np.zeros(n + 1, np.int64)
    off[1:] = np.cumsum([len(l) for l in nbrs])
    return {"x": x, "v": v, "material": mat, "nbr_off": off,
            "nbr_sets": np.concatenate([np.sort(l) for l in nbrs]).astype(np.int32) if off[-1] else np.zeros(0, np.int32),
            "density": density, "dfsph_factor": factor, "density_change": dchange, "acceleration": acc,
            "vorticity": vort, "grad_v": gradv, "kvn": kvn, "kden": kden, "omega": wt,
            "samples": samples.astype(np.int32), "v_vort": vv.astype(np.float64),
            "kden_sum_f32": np.array([kden_sum], F)}


if __name__ == "__main__":
    out = Path(__file__).resolve().parent
    for dim in (2, 3):
        data = run(dim, seed=7 + dim)
        np.savez_compressed(out / f"lattice{dim}d.npz", **data)
        print(dim, "d:", data["x"].shape[0], "particles,", data["nbr_off"][-1], "pairs")
