"""ctypes declarations of the C ABI in include/activechi4.h.

Loading fails loudly when the CUDA library has not been built: there is no
CPU fallback for the timestep.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libactivechi4_b200.so")

ACG_OK = 0
ACG_ERR_INVALID = -1
ACG_ERR_CUDA = -2
ACG_ERR_NOMEM = -3
ACG_ERR_NONFINITE = -4
ACG_ERR_STATE = -5
PREC_FP64 = 0
PREC_FP32 = 1


class acg_params(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("nact", C.c_int), ("L", C.c_double), ("density", C.c_double),
        ("T", C.c_double), ("f0", C.c_double), ("tau_p_steps", C.c_int), ("dt", C.c_double),
        ("skin", C.c_double), ("rebuild_factor", C.c_double), ("list_mode", C.c_int),
        ("thermostat", C.c_int), ("shuffle", C.c_int), ("precision", C.c_int),
        ("nb_capacity", C.c_int), ("seed", C.c_uint64), ("drift_every", C.c_int), ("P", C.c_double),
    ]


class acg_thermo(C.Structure):
    _fields_ = [
        ("pe", C.c_double), ("ke", C.c_double), ("virial", C.c_double), ("vir_act", C.c_double),
        ("inst_T", C.c_double), ("maxD", C.c_double), ("heff", C.c_double),
        ("eta", C.c_double * 3), ("p_eta", C.c_double * 3), ("q", C.c_double * 3),
        ("step", C.c_int64), ("rebuilds", C.c_int64), ("overflow", C.c_int), ("status", C.c_int),
        ("L", C.c_double), ("pressure", C.c_double), ("eps", C.c_double), ("p_eps", C.c_double),
        ("eta_baro", C.c_double * 3), ("p_eta_baro", C.c_double * 3),
    ]


class acg_obs_config(C.Structure):
    _fields_ = [
        ("run_length", C.c_int64), ("num_origins", C.c_int), ("factor", C.c_double),
        ("max_interval", C.c_int64), ("a", C.c_double), ("nq", C.c_int), ("qvec", C.c_void_p),
        ("max_live_origins", C.c_int),
    ]


class AcgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"activechi4 error {code}: {msg}")
        self.code = code


_lib = None

# name -> (restype, argtypes)
_SIGS = {
    "acg_params_default": (C.c_int, [C.POINTER(acg_params), C.c_int]),
    "acg_create": (C.c_int, [C.POINTER(acg_params), C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "acg_destroy": (C.c_int, [C.c_void_p]),
    "acg_footprint": (C.c_int, [C.POINTER(acg_params), C.c_int, C.POINTER(C.c_size_t)]),
    "acg_set_state": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "acg_get_state": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "acg_set_directions": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "acg_get_directions": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "acg_shuffle_directions": (C.c_int, [C.c_void_p, C.c_int]),
    "acg_seed_shuffle": (C.c_int, [C.c_void_p, C.c_int, C.c_uint64]),
    "acg_fix_drift": (C.c_int, [C.c_void_p, C.c_int]),
    "acg_adjust_temperature": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_double)]),
    "acg_start_ramp": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_int64)]),
    "acg_extend_ramp": (C.c_int, [C.c_void_p, C.c_int, C.c_int64]),
    "acg_set_lattice": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "acg_set_nhc": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "acg_set_barostat": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double]),
    "acg_set_temperature": (C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    "acg_rebuild": (C.c_int, [C.c_void_p]),
    "acg_compute_forces": (C.c_int, [C.c_void_p]),
    "acg_step": (C.c_int, [C.c_void_p, C.c_int]),
    "acg_step_eager": (C.c_int, [C.c_void_p, C.c_int]),
    "acg_sync": (C.c_int, [C.c_void_p]),
    "acg_poll": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "acg_get_thermo": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(acg_thermo)]),
    "acg_get_cells": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "acg_num_systems": (C.c_int, [C.c_void_p]),
    "acg_system_size": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "acg_stream": (C.c_void_p, [C.c_void_p]),
    "acg_set_priority": (C.c_int, [C.c_void_p, C.c_int]),
    "acg_release_retired": (C.c_int, []),
    "acg_prepare": (C.c_int, [C.c_void_p]),
    "acg_time_stage": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "acg_set_launch": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "acg_get_launch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "acg_set_group_tpp": (C.c_int, [C.c_void_p, C.c_int]),
    "acg_set_box_cells": (C.c_int, [C.c_void_p, C.c_int]),
    "acg_get_box_cells": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "acg_obs_configure": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(acg_obs_config)]),
    "acg_obs_sums": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "acg_bench_steps": (C.c_int, [C.c_void_p, C.c_int64, C.c_size_t, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "acg_measure_fp64_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    "acg_forces_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                     C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]),
    "acg_last_error": (C.c_char_p, []),
    "acg_version": (C.c_char_p, []),
}


def exported_symbols() -> list[str]:
    return list(_SIGS)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"activechi4 CUDA library not built ({LIB_PATH}); run "
                "`python -c 'import activechi4_b200.build as b; b.build()'` first")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != ACG_OK:
        raise AcgError(rc, lib().acg_last_error().decode())
