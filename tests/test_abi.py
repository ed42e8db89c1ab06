"""The C-ABI library loads on a CPU host, exports every symbol that
include/dimcv.h declares, and the ctypes structs match the C layout."""
import ctypes as C
import re

import numpy as np

from conftest import ROOT
from dimcv_sph_b200 import _abi, _lib


def declared_symbols():
    text = (ROOT / "include" / "dimcv.h").read_text()
    return sorted(set(re.findall(r"DV_API\s+[\w\s\*]+?\b(dv_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert len(names) >= 40
    for required in ("dv_create", "dv_grid_build", "dv_divergence_solve", "dv_pressure_solve",
                     "dv_vvpe_mc", "dv_bs_full", "dv_sample", "dv_akde"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()  # no GPU needed to load
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_prototypes_cover_header():
    assert set(declared_symbols()) == set(_lib.PROTOTYPES), \
        set(declared_symbols()) ^ set(_lib.PROTOTYPES)


def test_version_string_without_gpu():
    assert b"sm_100a" in _lib.load().dv_version()


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    lib = _lib.load()
    p = _abi.DvParams()
    p.dim = 5
    assert not lib.dv_create(C.byref(p), 10, None)
    assert b"dim" in lib.dv_last_error(None)


def test_struct_layout_matches_c():
    from oracle.oracle import load
    lib = load()
    lib.dvo_abi_layout.argtypes = [C.c_void_p]
    out = np.zeros(14, dtype=np.int64)
    lib.dvo_abi_layout(out.ctypes.data)
    assert out[0] == C.sizeof(_abi.DvParams)
    assert out[1] == C.sizeof(_abi.DvFields)
    assert out[2] == C.sizeof(_abi.DvSolverFields)
    assert out[3] == C.sizeof(_abi.DvCounters)
    assert out[4] == _abi.DvParams.eta_div.offset
    assert out[5] == _abi.DvParams.compensated.offset
    assert out[6] == _abi.DvCounters.err_div.offset
    assert out[7] == _abi.DvCounters.kden_sum_f32.offset
    assert out[8] == C.sizeof(_abi.DvVpmPlan)
    assert out[9] == C.sizeof(_abi.DvBatchScene)
    assert out[10] == _abi.DvBatchScene.seed.offset
    assert out[11] == C.sizeof(_abi.DvSceneState)
    assert out[12] == _abi.DvSceneState.err_div.offset
    assert out[13] == _abi.DvParams.n_scenes.offset
