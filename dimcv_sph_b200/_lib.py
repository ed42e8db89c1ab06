"""Loads libdimcv.so (the sm_100a CUDA library) and declares its C ABI.

There is no CPU fallback: if the shared library is missing or fails to load,
every entry point raises.  Build it with ``python -m dimcv_sph_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from ._abi import DvBatchScene, DvCounters, DvFields, DvParams, DvSceneState, DvSolverFields, DvVpmPlan

LIB_PATH = Path(os.environ.get("DIMCV_LIB", Path(__file__).resolve().parent / "libdimcv.so"))

_P = C.c_void_p
_FP = C.POINTER(DvFields)
_SP = C.POINTER(DvSolverFields)
_PP = C.POINTER(DvParams)
i32, i64, u64, f32, f64 = C.c_int32, C.c_int64, C.c_uint64, C.c_float, C.c_double

# name -> (restype, argtypes)
PROTOTYPES = {
    "dv_create": (_P, [_PP, i64, _P]),
    "dv_destroy": (None, [_P]),
    "dv_last_error": (C.c_char_p, [_P]),
    "dv_set_stream": (C.c_int, [_P, _P]),
    "dv_set_params": (C.c_int, [_P, _PP]),
    "dv_version": (C.c_char_p, []),
    "dv_launch_count": (i64, [_P]),
    "dv_get_counters": (C.c_int, [_P, C.POINTER(DvCounters)]),
    "dv_set_counts": (C.c_int, [_P, i32, i32, i32]),
    "dv_clear_status": (C.c_int, [_P]),
    "dv_add_particles": (C.c_int, [_P, _FP, _P, _P, i32, i32, f32, f32, i32, i32, i32, i32, i32, f32]),
    "dv_update_activity": (C.c_int, [_P, _FP]),
    "dv_grid_build": (C.c_int, [_P, _FP, _FP]),
    "dv_get_permutation": (C.c_int, [_P, C.POINTER(i32), i64]),
    "dv_neighbor_lists": (i64, [_P, _FP, _P, _P, i64]),
    "dv_stored_lists": (i64, [_P, _P, _P, i64]),
    "dv_boundary_volume": (C.c_int, [_P, _FP]),
    "dv_densities": (C.c_int, [_P, _FP]),
    "dv_dfsph_factor": (C.c_int, [_P, _FP]),
    "dv_densities_factor": (C.c_int, [_P, _FP]),
    "dv_densities_factor_change": (C.c_int, [_P, _FP]),
    "dv_scale_factor": (C.c_int, [_P, _FP, f32]),
    "dv_density_change": (C.c_int, [_P, _FP]),
    "dv_density_adv": (C.c_int, [_P, _FP]),
    "dv_density_error": (C.c_int, [_P, _FP, f32, C.POINTER(f64)]),
    "dv_divergence_iteration": (C.c_int, [_P, _FP]),
    "dv_pressure_iteration": (C.c_int, [_P, _FP]),
    "dv_divergence_solve": (C.c_int, [_P, _FP, C.POINTER(i32)]),
    "dv_divergence_solve_prepared": (C.c_int, [_P, _FP, C.POINTER(i32)]),
    "dv_divergence_solve_ex": (C.c_int, [_P, _FP, i32, C.POINTER(i32)]),
    "dv_pressure_solve_ex": (C.c_int, [_P, _FP, _SP, i32, C.POINTER(i32)]),
    "dv_pressure_solve": (C.c_int, [_P, _FP, C.POINTER(i32)]),
    "dv_nonpressure": (C.c_int, [_P, _FP]),
    "dv_predict_velocity": (C.c_int, [_P, _FP]),
    "dv_advect": (C.c_int, [_P, _FP]),
    "dv_moving_boundary_volume": (C.c_int, [_P, _FP]),
    "dv_set_dynamic_rigid": (C.c_int, [_P, C.c_int32]),
    "dv_enforce_boundary": (C.c_int, [_P, _FP, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "dv_dimcv_vorticity": (C.c_int, [_P, _FP, _SP]),
    "dv_d_vorticity": (C.c_int, [_P, _FP, _SP]),
    "dv_vorticity_dvort": (C.c_int, [_P, _FP, _SP]),
    "dv_smooth_akde": (C.c_int, [_P, _FP, _SP]),
    "dv_smooth_d_vort": (C.c_int, [_P, _FP, _SP]),
    "dv_kvn_sample": (C.c_int, [_P, _FP, _SP, u64, u64, i32]),
    "dv_record_samples": (C.c_int, [_P, _FP, _SP]),
    "dv_akde": (C.c_int, [_P, _FP, _SP]),
    "dv_sample": (C.c_int, [_P, _FP, _SP, i32, u64, u64, i32]),
    "dv_vvpe_mc": (C.c_int, [_P, _FP, _SP]),
    "dv_autotune": (C.c_int, [_P, _FP, _SP, C.POINTER(i32), C.POINTER(f32)]),
    "dv_set_far_tile": (C.c_int, [_P, i32]),
    "dv_life_time": (C.c_int, [_P, _FP]),
    "dv_vis": (C.c_int, [_P, _FP, _SP]),
    "dv_bs_full": (C.c_int, [_P, _FP, _P, _P, i32, _P, i32]),
    "dv_fp32_peak": (C.c_int, [_P, C.POINTER(f64)]),
    "dv_density_error_noalloc": (C.c_int, [_PP, _FP, i32, f32, C.POINTER(f64), _P]),
    "dv_profile": (C.c_int, [_P, i32]),
    "dv_set_far_chunks": (C.c_int, [_P, i32]),
    "dv_get_far_chunks": (i32, [_P]),
    "dv_vpm_workspace_bytes": (i64, [_P, i32, i32, i32]),
    "dv_batch_setup": (C.c_int, [_P, C.POINTER(DvBatchScene), i32, _P, i32, f32, i32]),
    "dv_batch_step": (C.c_int, [_P, _FP, _FP, _SP]),
    "dv_batch_graph_capture": (C.c_int, [_P, _FP, _FP, _SP, i32]),
    "dv_batch_graph_launch": (C.c_int, [_P]),
    "dv_batch_read": (C.c_int, [_P, C.POINTER(DvSceneState), i32, C.POINTER(i64)]),
    "dv_vpm_plan_build": (C.c_int, [_P, _FP, _SP, i32, C.POINTER(DvVpmPlan)]),
    "dv_vpm_smooth": (C.c_int, [_P, C.POINTER(DvVpmPlan), i32, _P, _P, _P]),
    "dv_vpm_curl": (C.c_int, [_P, C.POINTER(DvVpmPlan), i32, _P, _P, _P]),
    "dv_vpm_curl_bwd": (C.c_int, [_P, C.POINTER(DvVpmPlan), i32, _P, _P, _P, _P, _P]),
    "dv_vpm_smooth_bwd": (C.c_int, [_P, C.POINTER(DvVpmPlan), i32, _P, _P, _P, _P, _P]),
    "dv_vpm_velocity": (C.c_int, [_P, C.POINTER(DvVpmPlan), i32, _P, _P, _P, _P, i64]),
    "dv_vpm_velocity_bwd": (C.c_int, [_P, C.POINTER(DvVpmPlan), i32, _P, _P, _P, _P, _P, _P, i64]),
    "dv_profile_read": (C.c_int, [_P, C.POINTER(f64), C.POINTER(i64), C.POINTER(f64)]),
}

_lib = None


class DimcvError(RuntimeError):
    pass


def load():
    """Returns the loaded library, raising DimcvError if it is unavailable."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise DimcvError(
            f"{LIB_PATH} is missing: the CUDA library must be built "
            "(python -m dimcv_sph_b200.build); there is no CPU fallback")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(ctx, rc: int, what: str) -> int:
    if rc < 0:
        msg = load().dv_last_error(ctx)
        raise DimcvError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")
    return rc
