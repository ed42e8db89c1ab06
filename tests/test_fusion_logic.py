"""When the solver may skip a sweep that an earlier fused sweep already did
(host logic of DIMCVSPHSolver, no GPU): only while the library has launched
nothing since and torch has written none of the tensors the skipped sweep
reads, through any view."""
import torch

from dimcv_sph_b200.dimcv_sph import DIMCVSPHSolver


class _Lib:
    def __init__(self):
        self.launches = 0

    def dv_launch_count(self, ctx):
        return self.launches


class _Set:
    def __init__(self, names):
        self.t = {n: torch.zeros(8, 4) for n in names}

    def __getitem__(self, name):
        return self.t[name]


class _PS:
    def __init__(self):
        self.fields = _Set(("x", "v", "m", "m_V", "material", "vorticity", "density"))


def _solver():
    s = object.__new__(DIMCVSPHSolver)
    s.lib, s.ctx, s.ps = _Lib(), None, _PS()
    s._sb = {"v_star": torch.zeros(8, 4), "d_vort": torch.zeros(8, 4)}
    return s


def test_fresh_until_a_library_launch():
    s = _solver()
    mark = s._fusion_mark(s._CHANGE_READS)
    assert s._fusion_fresh(mark, s._CHANGE_READS)
    s.lib.launches += 1
    assert not s._fusion_fresh(mark, s._CHANGE_READS)


def test_in_place_edit_through_a_view_makes_it_stale():
    s = _solver()
    names = set(s._FACTOR_READS) | set(s._CHANGE_READS)
    mark = s._fusion_mark(names)
    view = s.ps.fields["v"][:, :3]
    view[:4] *= 1.5
    assert not s._fusion_fresh(mark, s._CHANGE_READS)  # the density change reads v
    assert s._fusion_fresh(mark, s._FACTOR_READS)      # the factor does not


def test_edit_of_an_unread_tensor_keeps_it_fresh():
    s = _solver()
    mark = s._fusion_mark(s._CHANGE_READS)
    s.ps.fields["density"].add_(1.0)
    assert s._fusion_fresh(mark, s._CHANGE_READS)


def test_solver_buffer_reads_are_tracked():
    s = _solver()
    mark = s._fusion_mark(s._DVORT_READS, ("v_star",))
    assert s._fusion_fresh(mark, s._DVORT_READS, ("v_star",))
    s._sb["d_vort"].fill_(2.0)  # written by the skipped sweep, not read
    assert s._fusion_fresh(mark, s._DVORT_READS, ("v_star",))
    s._sb["v_star"][0, 0] = 1.0
    assert not s._fusion_fresh(mark, s._DVORT_READS, ("v_star",))


def test_a_swapped_field_set_makes_it_stale():
    s = _solver()
    mark = s._fusion_mark(s._FACTOR_READS)
    s.ps.fields = _Set(("x", "v", "m", "m_V", "material", "vorticity", "density"))
    assert not s._fusion_fresh(mark, s._FACTOR_READS)


def test_no_mark_is_never_fresh():
    s = _solver()
    assert not s._fusion_fresh(None, s._FACTOR_READS)
