"""Scene batch: every scene of a batch step equals the same scene stepped
alone by the single-scene path (same cell grid, same initial slots, same
seed), CUDA-graph replay equals eager steps, and the per-scene bookkeeping
(counts, sample numbers, emission schedule, convergence) is consistent."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

FIELDS = ("x", "v", "density", "pressure", "dfsph_factor", "density_adv", "material", "m_V", "life_time")


@pytest.fixture(scope="module")
def small(cuda):
    from dimcv_sph_b200.batch import channel_batch_configs
    cfgs, _ = channel_batch_configs(n_scenes=4, seed=3, n_min=1500, n_max=4000, reserve_steps=60)
    return cfgs


def lone_run(cfg, grid_num, snap, counts, steps):
    """The scene on its own context, started from the batch's initial slots."""
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(cfg, grid_num=grid_num)
    sv = ps.build_solver()
    sv.far_tile = 4  # no autotuning: one sample chunk, as in the batch
    n, nf, ns = counts
    for k, t in snap.items():
        ps.fields[k][:n] = t
    ps.set_counts(n, nf, ns)
    for _ in range(steps):
        sv.step()
    return ps, sv


def test_batch_steps_equal_lone_scene_steps(small):
    from dimcv_sph_b200.batch import SceneBatch
    b = SceneBatch(small, keep_snapshots=True)
    steps = 3
    for _ in range(steps):
        b.step()
    st = b.states()
    for s, cfg in enumerate(small):
        ps, sv = lone_run(cfg, b.grid_num, b.snaps[s], b.snap_counts[s], steps)
        c = ps.counters()
        assert st[s]["end"] - st[s]["start"] == c["n"], s
        assert st[s]["n_fluid"] == c["n_fluid"] and st[s]["n_solid"] == c["n_solid"]
        assert st[s]["num_samples"] == c["num_samples"], s
        assert st[s]["iters_div"] == c["iters_div"] and st[s]["iters_p"] == c["iters_p"], s
        got = b.scene_fields(s, FIELDS, st)
        ref = {k: ps.fields[k][: c["n"]].cpu().numpy() for k in FIELDS}
        for k in FIELDS:
            assert np.array_equal(got[k], ref[k]), (s, k)
        sidx = sv.sample_idx[: c["num_samples"]].cpu().numpy()
        bidx = b.solver_buf["sample_idx"][st[s]["m_off"]: st[s]["m_off"] + st[s]["num_samples"]].cpu().numpy()
        assert np.array_equal(bidx - st[s]["start"], sidx), s


def test_graph_replay_equals_eager_steps(small):
    from dimcv_sph_b200.batch import SceneBatch
    a = SceneBatch(small)
    g = SceneBatch(small)
    for _ in range(2):
        a.step()
        g.step()
    g.capture(2)
    for _ in range(3):
        g.replay()
    for _ in range(6):
        a.step()
    torch.cuda.synchronize()
    assert g.steps == a.steps == 8
    sa, sg = a.states(), g.states()
    assert a.device_step == g.device_step == 8
    for s in range(a.S):
        fa = a.scene_fields(s, FIELDS, sa)
        fg = g.scene_fields(s, FIELDS, sg)
        for k in FIELDS:
            assert np.array_equal(fa[k], fg[k]), (s, k)
    assert sa == sg


def test_per_scene_bookkeeping(small):
    from dimcv_sph_b200.batch import SceneBatch
    b = SceneBatch(small)
    st0 = b.states()
    for _ in range(4):
        b.step()
    st = b.states()
    for s, info in enumerate(b.infos):
        # emission at steps 0 .. 3 of every scene whose interval divides them
        due = sum(1 for k in range(4) if info["emit_interval"] and k % info["emit_interval"] == 0)
        assert st[s]["emitted"] == due * info["emit_count"]
        nf = st[s]["n_fluid"]
        assert st[s]["num_samples"] == max(1, nf // 16)
        assert st[s]["n_targets"] == nf
        assert 1 <= st[s]["iters_p"] <= 100 and 1 <= st[s]["iters_div"] <= 100
        assert st[s]["kden_sum"] > 0
        assert st[s]["status"] & 0b11 == 0  # both solves converged
    # scenes are contiguous and ordered
    starts = [x["start"] for x in st]
    ends = [x["end"] for x in st]
    assert starts[0] == 0 and all(ends[s] == starts[s + 1] for s in range(b.S - 1))
    assert ends[-1] == b.counters()["n"]
    assert st0[0]["emitted"] == 0


def test_one_scene_batch_is_the_lone_run_in_a_graph(small):
    """A batch of one scene (no scene bits in the keys): eager steps equal the
    lone single-scene run bit for bit, and graph replays equal eager steps."""
    from dimcv_sph_b200.batch import SceneBatch
    b = SceneBatch(small[:1], keep_snapshots=True)
    for _ in range(3):
        b.step()
    st = b.states()
    ps, sv = lone_run(small[0], b.grid_num, b.snaps[0], b.snap_counts[0], 3)
    c = ps.counters()
    assert st[0]["start"] == 0 and st[0]["end"] == c["n"]
    got = b.scene_fields(0, FIELDS, st)
    for k in FIELDS:
        assert np.array_equal(got[k], ps.fields[k][: c["n"]].cpu().numpy()), k
    g = SceneBatch(small[:1])
    g.step()
    g.capture(2)
    g.replay()
    e = SceneBatch(small[:1])
    for _ in range(3):
        e.step()
    sg, se = g.states(), e.states()
    assert sg == se
    fg, fe = g.scene_fields(0, FIELDS, sg), e.scene_fields(0, FIELDS, se)
    for k in FIELDS:
        assert np.array_equal(fg[k], fe[k]), k


def test_more_scenes_than_the_ranked_block_order(cuda):
    """1,030 scenes, more than the 1,024 whose far-field blocks are issued
    longest first: the batch falls back to scene order, and scenes at both
    ends and in the middle still equal their lone runs."""
    from dimcv_sph_b200.batch import SceneBatch, channel_batch_configs
    cfgs, _ = channel_batch_configs(n_scenes=1030, seed=5, n_min=300, n_max=800, reserve_steps=20)
    b = SceneBatch(cfgs, keep_snapshots=True)
    steps = 2
    for _ in range(steps):
        b.step()
    st = b.states()
    for s in (0, 515, 1029):
        ps, sv = lone_run(cfgs[s], b.grid_num, b.snaps[s], b.snap_counts[s], steps)
        c = ps.counters()
        assert st[s]["end"] - st[s]["start"] == c["n"] and st[s]["num_samples"] == c["num_samples"], s
        got = b.scene_fields(s, FIELDS, st)
        for k in FIELDS:
            assert np.array_equal(got[k], ps.fields[k][: c["n"]].cpu().numpy()), (s, k)
