"""Pins the C++ oracle to the golden fixtures of the NumPy restatement
(tests/golden/make_golden.py) on jittered 2-D / 3-D lattices."""
import importlib.util

import numpy as np
import pytest

from conftest import ROOT
from dimcv_sph_b200.params import make_params
from oracle.oracle import OracleSim

_spec = importlib.util.spec_from_file_location("make_golden", ROOT / "tests" / "golden" / "make_golden.py")
make_golden = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(make_golden)


def relerr(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.max(np.abs(b)), 1e-30)
    return float(np.max(np.abs(a - b)) / scale)


def oracle_from_fixture(dim, order_mode):
    gold = dict(np.load(ROOT / "tests" / "golden" / f"lattice{dim}d.npz"))
    cfg, x, v, mat = make_golden.scene(dim, seed=7 + dim)
    assert np.array_equal(x, gold["x"]), "fixture is stale: rerun tests/golden/make_golden.py"
    p = make_params(cfg)
    n = x.shape[0]
    o = OracleSim(p, n + 8, order_mode)
    m_V0 = float(np.float32(0.8 * (2 * 0.01) ** dim))
    fl = mat == 1
    o.add_particles(x[fl], v[fl], 0, 1000.0, 0.0, 1, 1, (0, 0, 0), m_V0)
    o.add_particles(x[~fl], v[~fl], 1, 1000.0, 0.0, 0, 0, (0, 0, 0), m_V0)
    # input slot -> golden index: fluid first, then solids, each in order
    slot2gold = np.concatenate([np.nonzero(fl)[0], np.nonzero(~fl)[0]])
    o.initialize_particle_system()
    perm = o.permutation()
    g = slot2gold[perm]  # golden index of each sorted slot
    return o, gold, g


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order_mode", [0, 1])
def test_neighbour_sets_match_golden(dim, order_mode):
    o, gold, g = oracle_from_fixture(dim, order_mode)
    off, nbr = o.neighbor_lists()
    goff, gset = gold["nbr_off"], gold["nbr_sets"]
    for p in range(len(g)):
        mine = np.sort(g[nbr[off[p]:off[p + 1]]])
        ref = gset[goff[g[p]]:goff[g[p] + 1]]
        assert np.array_equal(mine, ref), (p, mine, ref)


@pytest.mark.parametrize("dim", [2, 3])
def test_sph_fields_match_golden(dim):
    o, gold, g = oracle_from_fixture(dim, 1)
    n = len(g)
    fl = gold["material"][g] == 1
    o.call("densities")
    o.call("dfsph_factor")
    o.call("density_change")
    o.call("nonpressure")
    o.calls("dimcv_vorticity")
    o.calls("kvn_sample", 0, 0, 0)
    o.calls("akde")
    f, s = o.f, o.solver
    assert relerr(f["density"][:n][fl], gold["density"][g][fl]) < 1e-6
    assert relerr(f["dfsph_factor"][:n][fl], gold["dfsph_factor"][g][fl]) < 1e-5
    assert relerr(f["density_adv"][:n][fl], gold["density_change"][g][fl]) < 1e-5
    assert relerr(f["acceleration"][:n, :dim][fl], gold["acceleration"][g][fl]) < 1e-5
    assert relerr(f["vorticity"][:n, :3][fl], gold["vorticity"][g][fl]) < 1e-5
    assert relerr(s["grad_v"][:n].reshape(n, dim, dim)[fl], gold["grad_v"][g][fl]) < 1e-5
    assert relerr(s["kvn"][:n][fl], gold["kvn"][g][fl]) < 1e-5
    assert relerr(s["kden"][:n][fl], gold["kden"][g][fl]) < 1e-5


@pytest.mark.parametrize("dim", [2, 3])
def test_vvpe_with_injected_samples_matches_golden(dim):
    o, gold, g = oracle_from_fixture(dim, 1)
    n = len(g)
    fl = gold["material"][g] == 1
    o.calls("dimcv_vorticity")
    o.calls("kvn_sample", 0, 0, 0)
    o.calls("akde")
    s = o.solver
    s["d_vort_smoothed"][:n, :3] = gold["omega"][g]
    inv = np.empty(n, np.int64)
    inv[g] = np.arange(n)
    smp = np.sort(inv[gold["samples"]]).astype(np.int32)
    s["sample_idx"][: len(smp)] = smp
    o.lib.dvo_set_num_samples(o.ctx, len(smp))
    # the FP64 sums are stored into the f32 v_vort field: 2^-24 rounding floor
    for prec, tol in ((64, 3e-7), (32, 1e-5)):
        o.calls("vvpe_mc", prec)
        got = s["v_vort"][:n, :3][fl].astype(np.float64)
        assert relerr(got, gold["v_vort"][g][fl]) < tol, prec
