"""The oracle against the reference's own outputs.

``tests/golden/reference_{channel2d,box3d}.npz`` hold what the unmodified
reference modules (``particle_system.py``, ``sph_base.py``, ``dimcv_sph.py``,
``karman_vortex.py``) computed on a 2-D channel and a 3-D box with the
reference's trimmed cylinder, two steps each, run through the serial Taichi
stand-in by ``tests/golden/make_reference_fixtures.py``.  The oracle runs in
the reference's visit order (order_mode 1: row-major cells, inclusive
prefix-sum ranges, flat cell 0 skipped), is loaded with the reference's
state before each step, and must reproduce every operator of
``KarmanVortexSolver.step`` (``karman_vortex.py:216-242``):

* partition + counting sort (``particle_system.py:413-560``): permutation,
  counts and every sorted field bit-exact;
* ``for_all_neighbors`` (``:562-586``): every list identical, in order;
* DFSPH, DIMCV and integration fields on fluid rows within 1e-5 normwise
  relative (``max|a-b| / max|b|``); ``d_vort`` = vorticity - curl(v*) and its
  smoothed form cancel to ~1e-3 of their operands, so their error is
  measured against max|vorticity|;
* Jacobi iteration counts, Bernoulli birth/death (``is_sample``, with the
  same Philox uniforms), sample lists and life times exactly;
* ``vort2vel``: the gate ``|v_vort| < |v|`` admits the same rows, v within
  1e-5, and the oracle's v_vort equals the reference's applied increment
  within 4 ulp of |v| (the reference keeps only the f32 sum v + v_vort).

The differences that remain (~1e-7) come from the two places where the
oracle and the reference round differently: ``r / |r| * h`` taken as one
reciprocal, and ``ti.pow(1 - q, 3.0)`` taken as a product.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from dimcv_sph_b200 import SimConfig
from dimcv_sph_b200._abi import vstride
from dimcv_sph_b200.params import make_params

GOLDEN = Path(__file__).resolve().parent / "golden"
SCENES = ("channel2d", "box3d")
RTOL = 1e-5

PS_LOAD = ("x", "v", "acceleration", "vorticity", "m_V", "m", "density", "pressure", "dfsph_factor",
           "density_adv", "life_time", "material", "object_id", "color", "is_dynamic", "is_active", "is_sample")


def _fixture(name):
    z = np.load(GOLDEN / f"reference_{name}.npz")
    meta = json.loads(bytes(z["meta"]).decode())
    scene = json.loads(bytes(z["scene_json"]).decode())
    return z, meta, scene


def _pad(a, k):
    a = np.asarray(a)
    if a.ndim == 1:
        return a
    out = np.zeros((a.shape[0], k), dtype=a.dtype)
    out[:, :a.shape[1]] = a
    return out


def _load(o, z, tag, dim):
    S = vstride(dim)
    comps = {"x": S, "v": S, "acceleration": S, "vorticity": 4, "color": 4}
    counts = z[f"{tag}/counts"]
    n = int(counts[0])
    snap = {f: _pad(z[f"{tag}/{f}"], comps.get(f, 1)) for f in PS_LOAD}
    for f, k in (("v_star", S), ("d_vort", 4), ("d_vort_smoothed", 4), ("x_temp", S)):
        snap["solver." + f] = _pad(z[f"{tag}/solver.{f}"], k)
    snap["solver.grad_v"] = z[f"{tag}/solver.grad_v"].reshape(n, -1)
    for f in ("kvn", "kden", "sample_idx"):
        snap["solver." + f] = z[f"{tag}/solver.{f}"]
    o.load_snapshot(snap, {"n": n, "n_fluid": int(counts[1]), "n_solid": int(counts[2]),
                           "num_samples": int(counts[3])})


def _rel(got, want):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    m = np.max(np.abs(want)) if want.size else 0.0
    d = np.max(np.abs(got - want)) if want.size else 0.0
    return d / m if m > 0 else d


def _cols(a, want):
    a = np.asarray(a)
    return a[:, :want.shape[1]] if a.ndim == 2 and np.asarray(want).ndim == 2 else a


@pytest.fixture(scope="module", params=SCENES)
def run(request):
    """Runs the oracle over every step of one fixture; returns the records."""
    from oracle.oracle import OracleSim
    name = request.param
    z, meta, scene = _fixture(name)
    dim = meta["dim"]
    P = make_params(SimConfig(config=scene))
    steps = []
    for k in range(meta["steps"]):
        rec = {"name": name, "step": k, "z": z, "meta": meta, "dim": dim, "checks": {}, "exact": {}}
        pre = f"s{k}/pre"
        o = OracleSim(P, int(z[f"{pre}/counts"][0]) + 64, order_mode=1)
        _load(o, z, pre, dim)
        o.update_activity()
        o.counting_sort()
        c = o.counters()
        n = c["n"]
        rec["exact"]["counts"] = ((c["n"], c["n_fluid"], c["n_solid"]), tuple(int(v) for v in z[f"s{k}/sorted/counts"]))
        g = o.snapshot()
        for f in ("x", "v", "acceleration", "m_V", "m", "density", "dfsph_factor", "density_adv", "life_time",
                  "material", "object_id", "is_dynamic", "is_sample"):
            rec["exact"]["sorted." + f] = (_cols(g[f], z[f"s{k}/sorted/{f}"]), z[f"s{k}/sorted/{f}"])
        off, nb = o.neighbor_lists()
        rec["exact"]["nbr_offsets"] = (off, z[f"s{k}/sorted/nbr_offsets"])
        rec["exact"]["nbr"] = (nb, z[f"s{k}/sorted/nbr"])
        fl = o.f["material"][:n] == 1
        rec["fluid"] = fl

        def check(stage, field, arr, want=None):
            want = z[f"s{k}/{stage}/{field}"] if want is None else want
            rec["checks"][f"{stage}.{field}"] = (_cols(np.array(arr[:n]), want)[fl], np.asarray(want)[fl])

        o.call("densities")
        check("compute_densities", "density", o.f["density"])
        o.call("dfsph_factor")
        check("compute_DFSPH_factor", "dfsph_factor", o.f["dfsph_factor"])
        it_div = o.divergence_solve()
        for f in ("v", "density_adv", "dfsph_factor"):
            check("divergence_solve", f, o.f[f])
        o.call("nonpressure")
        check("compute_non_pressure_forces", "acceleration", o.f["acceleration"])
        o.calls("dimcv_vorticity")
        check("compute_v_star", "v_star", o.solver["v_star"])
        check("compute_vorticity", "vorticity", o.f["vorticity"])
        check("compute_grad_v", "grad_v", o.solver["grad_v"], z[f"s{k}/compute_grad_v/grad_v"].reshape(n, -1))
        o.calls("d_vorticity")
        rec["d_vort"] = (o.solver["d_vort"][:n, :3].copy(), z[f"s{k}/compute_d_vorticity/d_vort"])
        o.calls("smooth_d_vort")
        rec["d_vort_smoothed"] = (o.solver["d_vort_smoothed"][:n, :3].copy(),
                                  z[f"s{k}/compute_all_d_vort_smoothed/d_vort_smoothed"])
        rec["vort_scale"] = float(np.max(np.abs(z[f"s{k}/compute_vorticity/vorticity"][fl])))
        o.calls("kvn_sample", meta["seed"], k, 1)
        check("compute_kinematic_vorticity_num_sample", "kinematic_vort_num", o.solver["kvn"])
        rec["exact"]["is_sample"] = (o.f["is_sample"][:n].copy(),
                                     z[f"s{k}/compute_kinematic_vorticity_num_sample/is_sample"])
        o.calls("record_samples")
        ns = o.counters()["num_samples"]
        rec["exact"]["sample_idx"] = (o.solver["sample_idx"][:ns].copy(),
                                      z[f"s{k}/record_vort_part_sample_idx/sample_idx"])
        inj_key = f"s{k}/record_vort_part_sample_idx/injected_idx"
        if inj_key in z:
            inj = z[inj_key]
            o.solver["sample_idx"][:inj.shape[0]] = inj
            o.lib.dvo_set_num_samples(o.ctx, int(inj.shape[0]))
            rec["injected"] = int(inj.shape[0])
        o.calls("akde")
        check("compute_kernel_density", "kernel_density", o.solver["kden"])
        rec["kden_sum"] = (o.counters()["kden_sum"], float(z[f"s{k}/compute_kernel_density/kden_sum"][0]))
        v_before = o.f["v"][:n].copy()
        o.calls("vvpe_mc", 32)
        check("vort2vel", "v", o.f["v"])
        rec["vvpe"] = (v_before, o.f["v"][:n].copy(), o.solver["v_vort"][:n].copy(),
                       z[f"s{k}/divergence_solve/v"], z[f"s{k}/vort2vel/v"])
        o.call("life_time")
        rec["exact"]["life_time"] = (o.f["life_time"][:n].copy(), z[f"s{k}/update_particle_life_time/life_time"])
        o.call("predict_velocity")
        check("predict_velocity", "v", o.f["v"])
        it_p = o.pressure_solve()
        rec["exact"]["iterations"] = ((it_div, it_p), tuple(meta["iterations"][k]))
        for f in ("v", "density_adv"):
            check("pressure_solve", f, o.f[f])
        o.calls("vis")
        rec["exact"]["x_temp"] = (_cols(o.solver["x_temp"][:n], z[f"s{k}/copy_x_temp/x_temp"]),
                                  z[f"s{k}/copy_x_temp/x_temp"])
        check("compute_vorticity_vis", "vorticity_vis", o.solver["vorticity_vis"])
        o.call("advect")
        check("advect", "x", o.f["x"])
        steps.append(rec)
    return steps


def test_fixtures_are_reference_runs():
    for name in SCENES:
        z, meta, scene = _fixture(name)
        assert meta["steps"] == 2 and meta["dim"] == len(scene["Configuration"]["domainStart"])
        assert all(f"s{k}/pre/x" in z for k in range(meta["steps"]))


def test_sort_and_neighbour_lists_bit_exact(run):
    for rec in run:
        for key, (got, want) in rec["exact"].items():
            if key.startswith("sorted.") or key.startswith("nbr") or key == "counts":
                if key == "counts":
                    assert got == want, (rec["name"], rec["step"], key)
                else:
                    assert np.array_equal(np.asarray(got), np.asarray(want)), (rec["name"], rec["step"], key)


def test_fields_within_tolerance(run):
    worst = {}
    for rec in run:
        for key, (got, want) in rec["checks"].items():
            e = _rel(got, want)
            worst[key] = max(worst.get(key, 0.0), e)
            assert e <= RTOL, (rec["name"], rec["step"], key, e)
    print({k: f"{v:.1e}" for k, v in worst.items()})


def test_vorticity_difference_within_tolerance_of_its_operands(run):
    for rec in run:
        fl = rec["fluid"]
        for key in ("d_vort", "d_vort_smoothed"):
            got, want = rec[key]
            e = np.max(np.abs(got[fl].astype(np.float64) - want[fl])) / rec["vort_scale"]
            assert e <= RTOL, (rec["name"], rec["step"], key, e)


def test_counts_samples_and_iterations_exact(run):
    for rec in run:
        for key in ("is_sample", "sample_idx", "life_time", "iterations", "x_temp"):
            got, want = rec["exact"][key]
            if key == "iterations":
                assert tuple(got) == tuple(want), (rec["name"], rec["step"], got, want)
            else:
                assert np.array_equal(np.asarray(got), np.asarray(want)), (rec["name"], rec["step"], key)
        s, s_ref = rec["kden_sum"]
        assert abs(s - s_ref) <= RTOL * abs(s_ref)


def test_vvpe_gate_and_increment(run):
    applied_total = 0
    for rec in run:
        dim = rec["dim"]
        vb, va, vv, vb_ref, va_ref = rec["vvpe"]
        app = np.any(va[:, :dim] != vb[:, :dim], axis=1)
        app_ref = np.any(va_ref != vb_ref, axis=1)
        assert np.array_equal(app, app_ref), (rec["name"], rec["step"])
        applied_total += int(app.sum())
        if app.any():
            inc_ref = (va_ref.astype(np.float64) - vb_ref)[app]
            ulp = np.spacing(np.float32(np.max(np.abs(va_ref))))
            err = np.max(np.abs(vv[app][:, :dim].astype(np.float64) - inc_ref))
            assert err <= 4 * ulp, (rec["name"], rec["step"], err, ulp)
    assert applied_total > 0


def test_ply_rows_match_the_reference_writer():
    """format_ply on the arrays the reference's export_ply read
    (karman_vortex.py:122-214, 3-D final frame) gives the same bytes."""
    from dimcv_sph_b200.export import format_ply
    z, meta, _ = _fixture("box3d")
    sets = meta["object_sets"]
    text = format_ply(z["ply/x_temp"], z["ply/vorticity"], z["ply/color"], z["ply/object_id"],
                      z["ply/is_active"], (sets["fluid_blocks"], sets["emitters"], sets["rigid_blocks"],
                                           sets["rigid_bodies"]))
    ref = bytes(z["ply/text"]).decode()
    assert text.splitlines()[:16] == ref.splitlines()[:16]
    assert text == ref
