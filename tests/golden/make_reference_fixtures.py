"""Golden fixtures from the reference's own code — TEST INFRASTRUCTURE ONLY.

Runs the unmodified reference modules (``particle_system.py``, ``sph_base.py``,
``dimcv_sph.py``, ``karman_vortex.py``, ``config_builder.py`` of
Haok-Z/DIMCV-SPH) on the CPU through the serial Taichi stand-in in
``ref_taichi/`` (trimesh and matplotlib, which the hot path never calls, are
empty modules), on two small scenes, and records what every operator of
``KarmanVortexSolver.step`` / ``substep`` (``karman_vortex.py:216-242``)
writes:

* ``channel2d``: a 2-D channel, 2 steps (about 750 particles);
* ``box3d``: a 3-D box with the reference's trimmed cylinder (object 2,
  ``karman_vortex.py:12-36``), 2 steps (about 1,600 particles).

The reference's own ``step()`` drives each run.  The script only wraps the
solver's methods on the instance to copy fields out after each call, counts
the Jacobi iterations, and sets the inputs:

* a swirl and a compression along x are added to the initial fluid
  velocity, so that every operator sees non-trivial data;
* ``ti.random`` (time-seeded in the reference, ``run_simulation.py:13``)
  returns Philox-4x32-10 uniforms keyed by (slot, step, seed) — the draws
  the oracle's Bernoulli sampler makes for the same slot (birth: word 0,
  death: word 1);
* in the second step the sample list that ``vort2vel`` reads is replaced by
  a fixed list (every 4th vortex-domain fluid slot) after
  ``record_vort_part_sample_idx``, so that the far field sums over enough
  samples.

For the 3-D scene the reference's ``export_ply`` also writes the final
frame, and the file's text is stored with the arrays it was written from.

Output: ``tests/golden/reference_<scene>.npz``.  Usage:

    python tests/golden/make_reference_fixtures.py [--reference DIR] [--scene NAME]

The reference directory is read here only; the tests read the committed
fixtures.
"""
from __future__ import annotations

import argparse
import io
import json
import sys
import time
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SEED = 0
N_STEPS = 2

FLUID_COLOR = [50, 100, 200]
SOLID_COLOR = [201, 112, 100]


def _block(obj, start, end, velocity, **extra):
    d = {"objectId": obj, "start": start, "end": end, "translation": [0.0] * len(start),
         "scale": [1] * len(start), "velocity": velocity, "density": 1000.0}
    d.update(extra)
    return d


SCENES = {
    "channel2d": {
        "Configuration": {
            "domainStart": [0.0, 0.0], "domainEnd": [1.0, 0.5], "particleRadius": 0.01,
            "numberOfStepsPerRenderUpdate": 1, "density0": 1000, "simulationMethod": 0,
            "gravitation": [0.0, 0.0], "timeStepSize": 0.0004, "bounceBackBoundary": False,
            "simulationTime": 1.0, "vortexEnforcingDomainStart": [0.2, 0.0],
            "vortexEnforcingDomainEnd": [1.0, 0.5], "volumeScale": 0.2, "GenProbPara": 5,
            "DelProbPara": 3.5, "reservedCapacity": 200, "divergenceTransitArea": [0.0, 0.02],
            "exportPLY": False},
        "FluidEmitters": [{"objectId": 0, "squareCenter": [0.0, 0.25], "squareSize": [0.0, 0.42],
                           "velocity": [1.0, 0.0], "density": 1000.0, "color": FLUID_COLOR}],
        "FluidBlocks": [_block(3, [0.02, 0.04], [0.5, 0.46], [1.0, 0.0], color=FLUID_COLOR)],
        "RigidBlocks": [
            _block(1, [0.0, 0.0], [1.0, 0.04], [0.0, 0.0], color=SOLID_COLOR, isDynamic=False),
            _block(1, [0.0, 0.46], [1.0, 0.5], [0.0, 0.0], color=SOLID_COLOR, isDynamic=False),
            _block(4, [0.6, 0.2], [0.68, 0.28], [0.0, 0.0], color=SOLID_COLOR, isDynamic=False),
        ],
    },
    "box3d": {
        "Configuration": {
            "domainStart": [0.0, 0.0, 0.0], "domainEnd": [1.0, 1.0, 0.28], "particleRadius": 0.02,
            "numberOfStepsPerRenderUpdate": 1, "density0": 1000, "simulationMethod": 0,
            "gravitation": [0.0, 0.0, -9.8], "timeStepSize": 0.004, "bounceBackBoundary": False,
            "simulationTime": 1.0, "vortexEnforcingDomainStart": [0.2, 0.0, 0.0],
            "vortexEnforcingDomainEnd": [1.0, 1.0, 0.28], "volumeScale": 0.2, "GenProbPara": 5,
            "DelProbPara": 3.5, "reservedCapacity": 200, "divergenceTransitArea": [0.0, 0.02, 0.02],
            "exportPLY": False},
        "FluidEmitters": [{"objectId": 0, "squareCenter": [0.0, 0.5, 0.14], "squareSize": [0.0, 0.8, 0.2],
                           "velocity": [1.0, 0.0, 0.0], "density": 1000.0, "color": FLUID_COLOR}],
        "FluidBlocks": [_block(3, [0.1, 0.1, 0.04], [0.5, 0.9, 0.24], [1.0, 0.0, 0.0], color=FLUID_COLOR)],
        "RigidBlocks": [
            _block(1, [0.0, 0.0, 0.0], [1.0, 0.04, 0.28], [0.0, 0.0, 0.0], color=SOLID_COLOR, isDynamic=False),
            _block(2, [0.5, 0.35, 0.04], [0.8, 0.65, 0.24], [0.0, 0.0, 0.0], color=SOLID_COLOR,
                   isDynamic=False),
        ],
    },
}

# particle fields recorded before each step (slots [0, particle_num))
PS_FIELDS = ("x", "v", "acceleration", "vorticity", "m_V", "m", "density", "pressure", "dfsph_factor",
             "density_adv", "life_time", "material", "object_id", "color", "is_dynamic", "is_active",
             "is_sample")
SOLVER_FIELDS = {"v_star": "v_star", "grad_v": "grad_v", "d_vort": "d_vort",
                 "d_vort_smoothed": "d_vort_smoothed", "kvn": "kinematic_vort_num",
                 "kden": "kernel_density", "x_temp": "x_temp", "sample_idx": "sample_idx"}

# what each tapped operator writes: (owner, field) pairs; owner "ps" or "solver"
STAGES = [
    ("compute_densities", [("ps", "density")]),
    ("compute_DFSPH_factor", [("ps", "dfsph_factor")]),
    ("divergence_solve", [("ps", "v"), ("ps", "density_adv"), ("ps", "dfsph_factor")]),
    ("compute_non_pressure_forces", [("ps", "acceleration")]),
    ("compute_v_star", [("solver", "v_star")]),
    ("compute_vorticity", [("ps", "vorticity")]),
    ("compute_grad_v", [("solver", "grad_v")]),
    ("compute_d_vorticity", [("solver", "d_vort")]),
    ("compute_all_d_vort_smoothed", [("solver", "d_vort_smoothed")]),
    ("compute_kinematic_vorticity_num_sample", [("solver", "kinematic_vort_num"), ("ps", "is_sample")]),
    ("record_vort_part_sample_idx", [("solver", "sample_idx")]),
    ("compute_kernel_density", [("solver", "kernel_density")]),
    ("vort2vel", [("ps", "v")]),
    ("update_particle_life_time", [("ps", "life_time")]),
    ("predict_velocity", [("ps", "v")]),
    ("pressure_solve", [("ps", "v"), ("ps", "density_adv")]),
    ("copy_x_temp", [("solver", "x_temp")]),
    ("compute_vorticity_vis", [("ps", "vorticity_vis")]),
    ("advect", [("ps", "x")]),
]


# ---------------------------------------------------------------- Philox
def philox4x32_10(c, k):
    """Philox-4x32-10 (Salmon et al., SC'11): counter c[4], key k[2] -> 4 words."""
    M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
    c0, c1, c2, c3 = c
    k0, k1 = k
    for _ in range(10):
        p0 = M0 * c0
        p1 = M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & 0xFFFFFFFF, p1 & 0xFFFFFFFF, \
            ((p0 >> 32) ^ c3 ^ k1) & 0xFFFFFFFF, p0 & 0xFFFFFFFF
        k0 = (k0 + W0) & 0xFFFFFFFF
        k1 = (k1 + W1) & 0xFFFFFFFF
    return c0, c1, c2, c3


def uniforms(slot, step, seed):
    o = philox4x32_10((slot, 0, step & 0xFFFFFFFF, step >> 32), (seed & 0xFFFFFFFF, seed >> 32))
    scale = np.float32(1.0 / 16777216.0)
    return np.float32(o[0] >> 8) * scale, np.float32(o[1] >> 8) * scale


# ---------------------------------------------------------------- driver
def import_reference(ref_dir: Path):
    sys.path.insert(0, str(HERE / "ref_taichi"))
    for name in ("trimesh", "matplotlib", "matplotlib.pyplot", "matplotlib.colors"):
        sys.modules[name] = types.ModuleType(name)
    sys.modules["matplotlib.colors"].Normalize = object
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    sys.modules["matplotlib"].colors = sys.modules["matplotlib.colors"]
    sys.path.insert(0, str(ref_dir))
    import taichi as ti  # the stand-in
    from config_builder import SimConfig
    from particle_system import ParticleSystem
    assert getattr(ti, "__version__", None) == (0, 0, 0), "the Taichi stand-in must shadow any real taichi"
    return ti, SimConfig, ParticleSystem


def run_scene(name: str, ref_dir: Path, tmp: Path) -> dict:
    ti, SimConfig, ParticleSystem = import_reference(ref_dir)
    scene = SCENES[name]
    path = tmp / f"{name}.json"
    path.write_text(json.dumps(scene))
    cfg = SimConfig(str(path))
    ps = ParticleSystem(cfg, GGUI=False)
    solver = ps.build_solver()
    dim = ps.dim
    out: dict[str, np.ndarray] = {}
    meta = {"scene": name, "dim": dim, "seed": SEED, "steps": N_STEPS, "iterations": [], "counts": []}

    # input: a swirl plus a compression along x on the initial fluid velocity
    n0 = ps.particle_num[None]
    x = ps.x.to_numpy()[:n0].astype(np.float64)
    fl = ps.material.to_numpy()[:n0] == ps.material_fluid
    L = np.array(scene["Configuration"]["domainEnd"], dtype=np.float64)
    sw = np.zeros_like(x)
    sw[:, 0] = 0.3 * np.sin(2 * np.pi * x[:, 1] / L[1]) + 0.2 * np.sin(2 * np.pi * x[:, 0] / L[0])
    sw[:, 1] = 0.3 * np.sin(2 * np.pi * x[:, 0] / L[0])
    v = ps.v.to_numpy()
    v[:n0][fl] += sw[fl].astype(np.float32)
    ps.v.from_numpy(v)

    state = {"step": -1, "div_iters": 0, "p_iters": 0}

    def rand_hook(loc):
        p_i = int(loc["p_i"])
        slf = loc["self"]
        u1, u2 = uniforms(p_i, state["step"], SEED)
        return u1 if slf.ps.is_sample.arr[p_i] == 0 else u2

    ti.set_random_hook(rand_hook)

    def grab(owner, fname, n):
        obj = ps if owner == "ps" else solver
        arr = getattr(obj, fname).arr
        return arr[:n].copy()

    def key(*parts):
        return "/".join(str(p) for p in parts)

    def record_state(tag):
        n = ps.particle_num[None]
        for f in PS_FIELDS:
            out[key(tag, f)] = grab("ps", f, n)
        for k, f in SOLVER_FIELDS.items():
            out[key(tag, "solver." + k)] = grab("solver", f, n)
        out[key(tag, "counts")] = np.array([n, ps.fluid_particle_num[None], ps.solid_particle_num[None],
                                            solver.num_samples[None]], dtype=np.int64)

    def neighbour_lists(n):
        offsets = np.zeros(n + 1, dtype=np.int64)
        nbrs = []

        def rec(p_i, p_j, ret):
            nbrs.append(int(p_j))

        with ti.kernel_scope():
            for i in range(n):
                ps.for_all_neighbors(i, rec, 0)
                offsets[i + 1] = len(nbrs)
        return offsets, np.array(nbrs, dtype=np.int32)

    # taps on the instance: the reference's step()/substep() call these
    orig_init_ps = ps.initialize_particle_system

    def init_ps_tap():
        if state["step"] >= 0:
            record_state(key("s%d" % state["step"], "pre"))
        orig_init_ps()
        if state["step"] >= 0:
            n = ps.particle_num[None]
            tag = key("s%d" % state["step"], "sorted")
            for f in PS_FIELDS:
                out[key(tag, f)] = grab("ps", f, n)
            out[key(tag, "counts")] = np.array([n, ps.fluid_particle_num[None], ps.solid_particle_num[None]],
                                               dtype=np.int64)
            off, nb = neighbour_lists(n)
            out[key(tag, "nbr_offsets")] = off
            out[key(tag, "nbr")] = nb

    ps.initialize_particle_system = init_ps_tap

    def make_tap(stage, fields):
        orig = getattr(solver, stage)

        def tap(*a, **k):
            r = orig(*a, **k)
            if state["step"] >= 0:
                n = ps.particle_num[None]
                tag = key("s%d" % state["step"], stage)
                for owner, f in fields:
                    out[key(tag, f)] = grab(owner, f, n)
                if stage == "record_vort_part_sample_idx":
                    ns = solver.num_samples[None]
                    out[key(tag, "num_samples")] = np.array([ns], dtype=np.int64)
                    out[key(tag, "sample_idx")] = solver.sample_idx.arr[:ns].copy()
                    if state["step"] == 1:  # injected sample list for the far field
                        inside = []
                        xs = ps.x.arr[:n]
                        mat = ps.material.arr[:n]
                        lo = scene["Configuration"]["vortexEnforcingDomainStart"]
                        hi = scene["Configuration"]["vortexEnforcingDomainEnd"]
                        for i in range(n):
                            if mat[i] == ps.material_fluid and all(
                                    lo[d] <= xs[i][d] <= hi[d] for d in range(dim)):
                                inside.append(i)
                        inj = np.array(inside[::4], dtype=np.int32)
                        solver.sample_idx.arr[:inj.shape[0]] = inj
                        solver.num_samples[None] = int(inj.shape[0])
                        out[key(tag, "injected_idx")] = inj
                if stage == "compute_kernel_density":
                    out[key(tag, "kden_sum")] = np.array([solver.kden_sum[None]], dtype=np.float32)
            return r

        setattr(solver, stage, tap)

    for stage, fields in STAGES:
        make_tap(stage, fields)

    orig_div_it = solver.divergence_solver_iteration
    orig_p_it = solver.pressure_solve_iteration

    def div_it():
        state["div_iters"] += 1
        return orig_div_it()

    def p_it():
        state["p_iters"] += 1
        return orig_p_it()

    solver.divergence_solver_iteration = div_it
    solver.pressure_solve_iteration = p_it

    # initial state (after ParticleSystem / KarmanVortexSolver construction)
    record_state("init")
    solver.initialize()
    record_state("initialized")
    meta["emit_interval"] = int(solver.emit_interval)
    for step in range(N_STEPS):
        state["step"] = step
        state["div_iters"] = state["p_iters"] = 0
        t0 = time.time()
        solver.step()
        meta["iterations"].append([state["div_iters"], state["p_iters"]])
        meta["counts"].append([ps.particle_num[None], ps.fluid_particle_num[None]])
        print(f"{name}: step {step} in {time.time() - t0:.1f} s, n={ps.particle_num[None]}, "
              f"iterations={meta['iterations'][-1]}, samples={solver.num_samples[None]}", flush=True)
    if dim == 3:
        # the reference's own PLY writer (karman_vortex.py:122-214) on the
        # final state, with the arrays it reads; its row loop unpacks three
        # coordinates, so it runs on 3-D scenes only
        solver.export_ply(N_STEPS - 1, tmp)
        out["ply/text"] = np.frombuffer((tmp / f"frame_{N_STEPS - 1:04}.ply").read_bytes(), dtype=np.uint8)
        n = ps.particle_num[None]
        out["ply/x_temp"] = solver.x_temp.arr[:n].copy()
        for f in ("vorticity", "color", "object_id", "is_active", "material"):
            out["ply/" + f] = getattr(ps, f).arr[:n].copy()
        meta["object_sets"] = {"emitters": sorted(ps.obj_id_emitters), "fluid_blocks": sorted(ps.obj_id_fluid_blocks),
                               "rigid_blocks": sorted(ps.obj_id_rigid_blocks),
                               "rigid_bodies": sorted(ps.object_id_rigid_body)}
    out["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    out["scene_json"] = np.frombuffer(json.dumps(scene).encode(), dtype=np.uint8)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--scene", default=None, choices=list(SCENES))
    ap.add_argument("--out", default=str(HERE))
    args = ap.parse_args()
    np.seterr(all="ignore")
    import tempfile
    for name in ([args.scene] if args.scene else list(SCENES)):
        with tempfile.TemporaryDirectory() as tmp:
            out = run_scene(name, Path(args.reference), Path(tmp))
        buf = io.BytesIO()
        np.savez_compressed(buf, **out)
        dst = Path(args.out) / f"reference_{name}.npz"
        dst.write_bytes(buf.getvalue())
        print(f"wrote {dst} ({dst.stat().st_size / 1024:.0f} KB)")


if __name__ == "__main__":
    main()
