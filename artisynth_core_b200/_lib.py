"""ctypes binding of libb200fem.so (C ABI in include/b200fem.h).

The shared library is the product: every compute call below goes to the
sm_100a kernels inside it.  There is no Python or CPU fallback -- if the
library is missing, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libb200fem.so")
HEADER = os.path.join(HERE, "..", "include", "b200fem.h")

OK = 0
ERR_INVALID_ARG = -1
ERR_CUDA = -2
ERR_STATE = -3
ERR_UNSUPPORTED = -4
ERR_INVERTED = -5
ERR_BUDGET = -6
ERR_TIMEOUT = -7
ERR_NO_CONVERGE = -13

ELEM_TET, ELEM_HEX, ELEM_WEDGE, ELEM_PYRAMID, ELEM_QUADTET, ELEM_QUADHEX, ELEM_QUADWEDGE, ELEM_QUADPYRAMID = range(8)
ELEM_NODES = {ELEM_TET: 4, ELEM_HEX: 8, ELEM_WEDGE: 6, ELEM_PYRAMID: 5, ELEM_QUADTET: 10, ELEM_QUADHEX: 20,
              ELEM_QUADWEDGE: 15, ELEM_QUADPYRAMID: 13}
MAT_LINEAR, MAT_NEOHOOKEAN, MAT_MOONEYRIVLIN, MAT_STVK = 0, 1, 2, 3
MAT_MODEL = -1  # b200fem_set_element_materials: the element keeps the model's material
INCOMP_OFF, INCOMP_NODAL, INCOMP_AUTO, INCOMP_ELEMENT = 0, 1, 2, 3
PREC_FP64, PREC_MIXED = 0, 1
PART_FULL, PART_UPPER = 0, 1
PCG_AUTO, PCG_CLASSIC, PCG_PIPELINED = 0, 1, 2
OPT_PCG_SPLIT, OPT_ROW_LANES, OPT_PCG_CTAS, OPT_PIECE_ROWS, OPT_WARM_START, OPT_ELEM_TILE, OPT_FUSED_ASSEMBLY = 1, 2, 3, 4, 5, 6, 7
OPT_REFINE = 8
OPT_BARRIER_TIMEOUT_MS, OPT_TEST_SKIP_ARRIVAL = 9, 10
OPT_TET_ASSEMBLY = 11
OPT_PCG_RESIDENT = 12
OPT_NODAL_FACTORED = 13
INTEGRATOR_BACKWARD_EULER, INTEGRATOR_CONSTRAINED_BACKWARD_EULER = 0, 1
SPLIT_AUTO, SPLIT_CONTIGUOUS, SPLIT_STRIDED, SPLIT_CLUSTER = 0, 1, 2, 3


class B200FemError(RuntimeError):
    """Raised for a non-zero status of a library call (cf. the reference's
    NumericalException from CuDssSolver.check, CuDssSolver.java:289-296)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"b200fem op failed (status {status}): {message}")
        self.status = status


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("precision", ctypes.c_int), ("reserved", ctypes.c_int * 6)]


class StepParams(ctypes.Structure):
    _fields_ = [
        ("h", ctypes.c_double),
        ("alpha_m", ctypes.c_double),
        ("beta_k", ctypes.c_double),
        ("gravity", ctypes.c_double * 3),
        ("tol", ctypes.c_double),
        ("max_iter", ctypes.c_int),
        ("abort_on_inverted", ctypes.c_int),
        ("pcg_variant", ctypes.c_int),
        ("integrator", ctypes.c_int),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("num_inverted", ctypes.c_int),
        ("rel_residual", ctypes.c_double),
        ("min_detJ", ctypes.c_double),
        ("refinements", ctypes.c_int),
        ("reserved", ctypes.c_int * 3),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("ticks", ctypes.c_longlong), ("model_steps", ctypes.c_longlong), ("slot_steps", ctypes.c_longlong),
        ("builds", ctypes.c_longlong), ("evictions", ctypes.c_longlong), ("completed", ctypes.c_longlong),
        ("failed", ctypes.c_longlong), ("resident_bytes", ctypes.c_ulonglong), ("peak_bytes", ctypes.c_ulonglong),
        ("pending", ctypes.c_int), ("resident_models", ctypes.c_int),
    ]


_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


def header_symbols() -> list[str]:
    """Names of every function declared in include/b200fem.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(b200fem_[a-z0-9_]+)\s*\(", text)))


def lib():
    """Load libb200fem.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m artisynth_core_b200.build` "
            "(the engine has no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    H = _vp
    sig = {
        "b200fem_version": ([], ctypes.c_int),
        "b200fem_create": ([ctypes.POINTER(Config)], H),
        "b200fem_destroy": ([H], ctypes.c_int),
        "b200fem_last_error": ([H], ctypes.c_char_p),
        "b200fem_grid_dims": ([ctypes.c_int] * 4 + [_ip, _ip], ctypes.c_int),
        "b200fem_create_grid": ([ctypes.c_int] + [ctypes.c_double] * 3 + [ctypes.c_int] * 3 + [_dp, _ip], ctypes.c_int),
        "b200fem_jitter_grid": ([ctypes.c_int] * 3 + [ctypes.c_double] * 4 + [ctypes.c_ulonglong, _dp], ctypes.c_int),
        "b200fem_quadratic_tet_mesh": ([ctypes.c_int, _dp, ctypes.c_int, _ip, ctypes.POINTER(ctypes.c_int), _dp, _ip],
                                       ctypes.c_int),
        "b200fem_set_mesh": ([H, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _ip, _ip], ctypes.c_int),
        "b200fem_set_mesh_mixed": ([H, ctypes.c_int, _dp, ctypes.c_int, _ip, _ip, _ip], ctypes.c_int),
        "b200fem_set_material": ([H, ctypes.c_int, _dp, ctypes.c_double, ctypes.c_int], ctypes.c_int),
        "b200fem_set_element_materials": ([H, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
                                          ctypes.c_int),
        "b200fem_build": ([H], ctypes.c_int),
        "b200fem_get_sizes": ([H, _ip, _ip, _ip, _ip], ctypes.c_int),
        "b200fem_get_solve_index": ([H, _ip], ctypes.c_int),
        "b200fem_get_pattern": ([H, _ip, _ip], ctypes.c_int),
        "b200fem_get_crs_indices": ([H, ctypes.c_int, _ip, _ip], ctypes.c_int),
        "b200fem_get_slot_map": ([H, ctypes.c_int, _ip], ctypes.c_int),
        "b200fem_get_scatter_map": ([H, _ip], ctypes.c_int),
        "b200fem_get_masses": ([H, _dp], ctypes.c_int),
        "b200fem_get_incomp_method": ([H, _ip], ctypes.c_int),
        "b200fem_set_state": ([H, _dp, _dp], ctypes.c_int),
        "b200fem_get_state": ([H, _dp, _dp], ctypes.c_int),
        "b200fem_set_external_forces": ([H, _dp], ctypes.c_int),
        "b200fem_update_stress_stiffness": ([H, _dp, _dp, _dp, _dp], ctypes.c_int),
        "b200fem_backward_euler_step": ([H, ctypes.POINTER(StepParams), ctypes.c_int, ctypes.POINTER(Stats)], ctypes.c_int),
        "b200fem_set_plane_constraints": ([H, ctypes.c_int, _ip, _dp, _dp], ctypes.c_int),
        "b200fem_set_frame_attachments": ([H, ctypes.c_int, ctypes.c_int, _ip, _ip, _dp], ctypes.c_int),
        "b200fem_set_point_constraints": ([H, ctypes.c_int, _ip, _ip, _dp, _dp], ctypes.c_int),
        "b200fem_backward_euler_step_host": ([H, ctypes.POINTER(StepParams), ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.POINTER(Stats)], ctypes.c_int),
        "b200fem_spmv": ([H, _dp, _dp], ctypes.c_int),
        "b200fem_pcg_solve": ([H, _dp, _dp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(Stats)], ctypes.c_int),
        "b200fem_last_timing": ([H, _dp, _dp], ctypes.c_int),
        "b200fem_add_model": ([H, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _ip, _ip, ctypes.c_int, _dp,
                               ctypes.c_double, ctypes.c_int, _ip], ctypes.c_int),
        "b200fem_clear_models": ([H], ctypes.c_int),
        "b200fem_num_models": ([H, _ip], ctypes.c_int),
        "b200fem_model_range": ([H, ctypes.c_int, _ip, _ip, _ip], ctypes.c_int),
        "b200fem_get_model_stats": ([H, _ip, _dp], ctypes.c_int),
        "b200fem_set_option": ([H, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "b200fem_set_active_models": ([H, _ip], ctypes.c_int),
        "b200fem_memory_usage": ([H, ctypes.POINTER(ctypes.c_ulonglong)], ctypes.c_int),
        "b200fem_get_option": ([H, ctypes.c_int, _ip], ctypes.c_int),
        "b200fem_server_create": ([ctypes.POINTER(Config), ctypes.c_double, ctypes.c_int,
                                   ctypes.POINTER(StepParams)], H),
        "b200fem_server_destroy": ([H], ctypes.c_int),
        "b200fem_server_last_error": ([H], ctypes.c_char_p),
        "b200fem_server_clock": ([H], ctypes.c_double),
        "b200fem_server_set_option": ([H, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "b200fem_server_add_model": ([H, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _ip, _ip, ctypes.c_int,
                                      _dp, ctypes.c_double, ctypes.c_int, _dp, _ip], ctypes.c_int),
        "b200fem_server_submit": ([H, ctypes.c_int, ctypes.c_int, ctypes.c_double, _ip], ctypes.c_int),
        "b200fem_server_preload": ([H], ctypes.c_int),
        "b200fem_server_tick": ([H, _ip], ctypes.c_int),
        "b200fem_server_poll": ([H, ctypes.c_int, _ip, _dp], ctypes.c_int),
        "b200fem_server_get_state": ([H, ctypes.c_int, _dp, _dp], ctypes.c_int),
        "b200fem_server_get_stats": ([H, ctypes.POINTER(ServerStats)], ctypes.c_int),
        "b200fem_pcg_solve_noalloc": ([ctypes.c_int, _vp, _vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_int, _vp,
                                       _ip, _dp], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def dptr(a):
    """double* of a C-contiguous float64 array (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def iptr(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def check(status: int, handle=None):
    if status != OK:
        msg = lib().b200fem_last_error(handle)
        raise B200FemError(status, (msg or b"").decode(errors="replace"))
    return status
