"""The device-side step paths against the oracle, step by step.

Two paths step scenes with no host work inside a step: a batch of scenes
(one launch per stage for all of them, device emission, device Jacobi loops)
and a batch of one scene replayed from a CUDA graph.  Each is compared with
the oracle: before every compared step the oracle is loaded with the scene's
slots as the device left them, then runs the step itself (the emission when
it is due, ``dimcv_sph.py:616-637`` with ``particle_system.py:334-380``; the
activity update and grid build; the substep with the same inverse-CDF
draws).  After the step the fluid x, v and DFSPH fields agree within 1e-5
(the far field is FP64 in the oracle), the samples and Jacobi iteration
counts are identical.

* 4 scenes of 1.5k-4k particles, 34 steps: every scene emits at step 0 and
  once more (intervals of 27-32 steps);
* the 1-scene graph: 2 steps per replay, 15 replays (30 steps), the oracle
  stepping twice per reload.
"""
import numpy as np
import pytest

from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu

RTOL = 1e-5
KEYS = ("x", "v", "density", "density_adv", "dfsph_factor")


def _relerr(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


@pytest.fixture(scope="module")
def cfgs(cuda):
    from dimcv_sph_b200.batch import channel_batch_configs
    c, _ = channel_batch_configs(n_scenes=4, seed=9, n_min=1500, n_max=4000, reserve_steps=60)
    return c


def _scene_params(cfg, grid_num):
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(cfg, grid_num=grid_num)
    return ps.params, int(ps.particle_max_num)


def _load_scene(b, s, st, params, cap):
    """An oracle holding scene s's slots (scene-local, in the batch's order)."""
    a, e = st[s]["start"], st[s]["end"]
    o = OracleSim(params, cap, 0)
    snap = {k: t[a:e].cpu().numpy() for k, t in b.fields.t.items()}
    snap.update({"solver." + k: t[a:e].cpu().numpy() for k, t in b.solver_buf.t.items() if k != "sample_idx"})
    o.load_snapshot(snap, {"n": e - a, "n_fluid": st[s]["n_fluid"], "n_solid": st[s]["n_solid"]})
    return o


def _oracle_step(o, b, s, step):
    """KarmanVortexSolver.step on the oracle (emission when due)."""
    info = b.infos[s]
    if info["emit_interval"] and step % info["emit_interval"] == 0:
        pos = b._emit[info["emit_offset"]: info["emit_offset"] + info["emit_count"]]
        vel = np.tile(np.asarray(info["emit_velocity"][:2], np.float32), (pos.shape[0], 1))
        o.add_particles(pos, vel, s, float(np.float32(info["emit_density"])), 0.0, 1, 1,
                        tuple(info["emit_color"]), float(np.float32(info["m_V0"])))
    o.update_activity()
    o.counting_sort()
    M = max(1, o.counters()["n_fluid"] // 16)
    it = o.substep(seed=info["seed"], step=step, sampler="inverse_cdf", M=M, compute_vis=False,
                   vvpe_precision=64)
    return M, it


def _compare(b, s, st, o, M, it, tag):
    a, e = st[s]["start"], st[s]["end"]
    c = o.counters()
    assert e - a == c["n"] and st[s]["n_fluid"] == c["n_fluid"], tag
    r = o.snapshot()
    g = {k: b.fields[k][a:e].cpu().numpy() for k in KEYS + ("material",)}
    fl = g["material"] == 1
    worst = {}
    for k in KEYS:
        worst[k] = _relerr(g[k][fl], r[k][fl])
        assert worst[k] < RTOL, (tag, k, worst[k])
    assert st[s]["num_samples"] == M, tag
    bidx = b.solver_buf["sample_idx"][st[s]["m_off"]: st[s]["m_off"] + M].cpu().numpy() - a
    assert np.array_equal(bidx, r["solver.sample_idx"][:M]), tag
    assert (st[s]["iters_div"], st[s]["iters_p"]) == tuple(it), tag
    return worst


def _initial_states(b):
    """Scene ranges of the batch as built (the device states are set by the
    first step): scenes in order, each with its initial counts."""
    st, o = [], 0
    for n, nf, ns in b.snap_counts:
        st.append({"start": o, "end": o + n, "n_fluid": nf, "n_solid": ns})
        o += n
    return st


def test_scene_batch_matches_oracle_every_step(cfgs):
    from dimcv_sph_b200.batch import SceneBatch
    b = SceneBatch(cfgs, keep_snapshots=True)
    params = [_scene_params(c, b.grid_num) for c in cfgs]
    st = _initial_states(b)
    for step in range(34):
        oracles = [_load_scene(b, s, st, *params[s]) for s in range(b.S)]
        b.step()
        st = b.states()
        for s in range(b.S):
            M, it = _oracle_step(oracles[s], b, s, step)
            _compare(b, s, st, oracles[s], M, it, (s, step))
    for s, info in enumerate(b.infos):
        assert st[s]["emitted"] == 2 * info["emit_count"], s  # step 0 and once more


def test_one_scene_graph_matches_oracle(cfgs):
    from dimcv_sph_b200.batch import SceneBatch
    b = SceneBatch(cfgs[1:2], keep_snapshots=True)
    params = _scene_params(cfgs[1], b.grid_num)
    b.capture(2)
    st = _initial_states(b)
    step = 0
    for _ in range(15):
        o = _load_scene(b, 0, st, *params)
        b.replay()
        st = b.states()
        for _k in range(2):
            M, it = _oracle_step(o, b, 0, step)
            step += 1
        _compare(b, 0, st, o, M, it, step)
    assert st[0]["emitted"] == 2 * b.infos[0]["emit_count"]
