"""ctypes mirror of include/dimcv.h (structs and constants only).

Importable without a GPU or the CUDA library: the CPU oracle wrapper and the
host-side parameter code share these definitions with the CUDA binding.
"""
from __future__ import annotations

import ctypes as C

DV_OK = 0
DV_EINVAL = -1
DV_ECAPACITY = -2
DV_ECUDA = -3
DV_ENAN = -4
DV_EUNSUPPORTED = -5

DV_WARN_DIV_NOT_CONVERGED = 1 << 0
DV_WARN_P_NOT_CONVERGED = 1 << 1
DV_WARN_OUTSIDE_GRID = 1 << 2
DV_WARN_CAPACITY = 1 << 3
DV_WARN_NAN = 1 << 4
DV_WARN_BAD_INDEX = 1 << 5

DV_SAMPLE_BERNOULLI = 0
DV_SAMPLE_INVERSE_CDF = 1
DV_SAMPLE_INJECTED = 2
DV_SAMPLE_STRATIFIED = 3

DV_SOLVE_PREPARED = 1
DV_SOLVE_NONPRESSURE = 2
DV_SOLVE_VIS = 4

DV_KERNEL_REF2D = 0
DV_KERNEL_BLOB3D = 1

DV_VPM_MC = 0
DV_VPM_FULL = 1

MATERIAL_SOLID = 0
MATERIAL_FLUID = 1

F3 = C.c_float * 3
I3 = C.c_int32 * 3


class DvParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int32),
        ("grid_num", I3),
        ("domain_start", F3),
        ("domain_end", F3),
        ("grid_size", C.c_float),
        ("support_radius", C.c_float),
        ("inv_support_radius", C.c_float),
        ("nbr_r2_limit", C.c_float),
        ("far_r2_limit", C.c_float),
        ("kW", C.c_float),
        ("kW2", C.c_float),
        ("kG", C.c_float),
        ("grad_r_min", C.c_float),
        ("density0", C.c_float),
        ("dt", C.c_float),
        ("inv_dt", C.c_float),
        ("inv_dt2", C.c_float),
        ("gravity", F3),
        ("visc_coef", C.c_float),
        ("visc_h2", C.c_float),
        ("m_eps", C.c_float),
        ("factor_min", C.c_float),
        ("eta_div", C.c_double),
        ("eta_p", C.c_double),
        ("max_iter_div", C.c_int32),
        ("max_iter_p", C.c_int32),
        ("neighbor_min", C.c_int32),
        ("has_transit", C.c_int32),
        ("transit_a0", C.c_float),
        ("transit_span", C.c_float),
        ("has_vortex_domain", C.c_int32),
        ("vd_start", F3),
        ("vd_end", F3),
        ("vvpe_coef", C.c_float),
        ("eps", C.c_float),
        ("inv_eps", C.c_float),
        ("gen_a", C.c_float),
        ("del_b", C.c_float),
        ("kden_eps", C.c_float),
        ("kvn_eps", C.c_float),
        ("skip_cell0", C.c_int32),
        ("cell_origin_offset", C.c_int32),
        ("kernel_mode", C.c_int32),
        ("blob_delta2", C.c_float),
        ("blob_coef", C.c_float),
        ("compensated", C.c_int32),
        ("periodic", C.c_int32),
        ("box", F3),
        ("n_scenes", C.c_int32),
        ("reserved", C.c_int32 * 3),
    ]


_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int32)
_BP = C.POINTER(C.c_uint8)


class DvFields(C.Structure):
    _fields_ = [
        ("x", _FP), ("x0", _FP), ("v", _FP), ("acceleration", _FP),
        ("vorticity", _FP),
        ("m_V", _FP), ("m", _FP), ("density", _FP), ("pressure", _FP),
        ("dfsph_factor", _FP), ("density_adv", _FP), ("life_time", _FP),
        ("material", _IP), ("object_id", _IP), ("color", _IP), ("grid_ids", _IP),
        ("is_dynamic", _BP), ("is_active", _BP), ("is_sample", _BP),
    ]


class DvSolverFields(C.Structure):
    _fields_ = [
        ("v_star", _FP), ("grad_v", _FP), ("d_vort", _FP), ("d_vort_smoothed", _FP),
        ("kvn", _FP), ("kden", _FP), ("x_temp", _FP), ("vorticity_vis", _FP),
        ("v_vort", _FP), ("sample_idx", _IP),
    ]


class DvVpmPlan(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("src_cap", C.c_int32), ("nbr_cap", C.c_int64),
        ("n_src", C.c_void_p), ("perm", C.c_void_p), ("inv_perm", C.c_void_p),
        ("nbr_off", C.c_void_p), ("nbr", C.c_void_p), ("src", C.c_void_p), ("src_a", C.c_void_p),
        ("slot_src", C.c_void_p), ("slot_a", C.c_void_p), ("f", C.c_void_p), ("m_V", C.c_void_p),
        ("xbar", C.c_void_p),
    ]


class DvBatchScene(C.Structure):
    _fields_ = [
        ("domain_end", F3), ("cap", C.c_int32), ("emit_offset", C.c_int32), ("emit_count", C.c_int32),
        ("emit_interval", C.c_int32), ("emit_velocity", F3), ("emit_density", C.c_float),
        ("emit_color", I3), ("emit_volume", C.c_float), ("pad", C.c_int32), ("seed", C.c_uint64),
    ]


class DvSceneState(C.Structure):
    _fields_ = [
        ("start", C.c_int32), ("end", C.c_int32), ("n_fluid", C.c_int32), ("n_solid", C.c_int32),
        ("t_start", C.c_int32), ("n_targets", C.c_int32), ("m_off", C.c_int32), ("num_samples", C.c_int32),
        ("tile_off", C.c_int32), ("iters_div", C.c_int32), ("iters_p", C.c_int32), ("done", C.c_int32),
        ("status", C.c_int32), ("emitted", C.c_int32),
        ("err_div", C.c_double), ("err_p", C.c_double), ("kden_sum", C.c_double),
        ("kden_sum_f32", C.c_float), ("pad", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class DvCounters(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("n_fluid", C.c_int32), ("n_solid", C.c_int32),
        ("num_samples", C.c_int32), ("iters_div", C.c_int32), ("iters_p", C.c_int32),
        ("status", C.c_int32), ("n_targets", C.c_int32),
        ("err_div", C.c_double), ("err_p", C.c_double), ("kden_sum", C.c_double),
        ("kden_sum_f32", C.c_float), ("pad", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


# field name -> (dtype, components per particle) ; 'S' = DV_VSTRIDE(dim)
PARTICLE_FIELDS = {
    "x": ("f32", "S"), "x0": ("f32", "S"), "v": ("f32", "S"), "acceleration": ("f32", "S"),
    "vorticity": ("f32", 4),
    "m_V": ("f32", 1), "m": ("f32", 1), "density": ("f32", 1), "pressure": ("f32", 1),
    "dfsph_factor": ("f32", 1), "density_adv": ("f32", 1), "life_time": ("f32", 1),
    "material": ("i32", 1), "object_id": ("i32", 1), "color": ("i32", 4), "grid_ids": ("i32", 1),
    "is_dynamic": ("u8", 1), "is_active": ("u8", 1), "is_sample": ("u8", 1),
}
SOLVER_FIELDS = {
    "v_star": ("f32", "S"), "grad_v": ("f32", "DD"), "d_vort": ("f32", 4),
    "d_vort_smoothed": ("f32", 4), "kvn": ("f32", 1), "kden": ("f32", 1),
    "x_temp": ("f32", "S"), "vorticity_vis": ("f32", 4), "v_vort": ("f32", 4),
    "sample_idx": ("i32", 1),
}


def vstride(dim: int) -> int:
    return 2 if dim == 2 else 4


def components(spec, dim: int) -> int:
    if spec == "S":
        return vstride(dim)
    if spec == "DD":
        return dim * dim
    return int(spec)


_PTR_T = {"f32": _FP, "i32": _IP, "u8": _BP}


def make_struct(cls, ptrs: dict):
    """Builds a DvFields / DvSolverFields from {name: integer address}."""
    s = cls()
    for name, typ in cls._fields_:
        addr = ptrs.get(name, 0)
        setattr(s, name, C.cast(C.c_void_p(addr), typ) if addr else typ())
    return s
