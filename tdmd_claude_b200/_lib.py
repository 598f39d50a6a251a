"""ctypes binding of the C ABI in include/tdmd_b200.h (libtdmd_b200.so).

The shared library is built in-tree (tdmd_claude_b200/build.py).  There is
no fallback: if the library is missing or fails to load, every entry point
raises -- the product path is the CUDA library or nothing.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtdmd_b200.so")

TDMD_OK = 0
TDMD_FP64 = 0
TDMD_MIXED = 1
TDMD_POT_MORSE = 0
TDMD_POT_EAM = 1

STATUS_NAMES = {
    0: "OK", 1: "INVALID_ARGUMENT", 2: "CUDA", 3: "OUT_OF_MEMORY", 4: "PARSE", 5: "STATE",
    6: "NLIST_OVERFLOW", 7: "TIMEOUT", 8: "UNSUPPORTED", 9: "IO",
}


class TdmdError(RuntimeError):
    """Non-zero tdmd_status from the C ABI (mirrors tdmd::Error)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{STATUS_NAMES.get(code, code)}] {msg}")
        self.code = code


class Box(C.Structure):
    """tdmd_box -- Box, src/core/box.hpp:17."""
    _fields_ = [("lo", C.c_double * 3), ("hi", C.c_double * 3), ("periodic", C.c_int32 * 3)]

    @classmethod
    def make(cls, lo, hi, periodic=(True, True, True)):
        b = cls()
        for a in range(3):
            b.lo[a] = float(lo[a])
            b.hi[a] = float(hi[a])
            b.periodic[a] = 1 if periodic[a] else 0
        return b

    def size(self):
        return tuple(self.hi[a] - self.lo[a] for a in range(3))


class MorseParams(C.Structure):
    """tdmd_morse_params -- MorseParams, src/potentials/device_morse.cuh:14."""
    _fields_ = [("d", C.c_double), ("alpha", C.c_double), ("r0", C.c_double), ("rc", C.c_double),
                ("rc_sq", C.c_double)]

    @classmethod
    def make(cls, d, alpha, r0, rc):
        return cls(float(d), float(alpha), float(r0), float(rc), float(rc) * float(rc))


class FastPipelineConfig(C.Structure):
    """tdmd_fast_pipeline_config -- FastPipelineConfig (+ precision, NVT, ...)."""
    _fields_ = [("dt", C.c_double), ("r_skin", C.c_double), ("rebuild_every", C.c_int32),
                ("precision", C.c_int32), ("use_graphs", C.c_int32),
                ("lanes_per_atom", C.c_int32), ("t_target", C.c_double),
                ("t_period", C.c_double), ("nhc_length", C.c_int32), ("adaptive_dt", C.c_int32),
                ("dt_min", C.c_double), ("dt_max", C.c_double), ("c2", C.c_double),
                ("energy_every", C.c_int32), ("energy_log_capacity", C.c_int32),
                ("nbr_batch", C.c_int32)]


class FastPipelineStats(C.Structure):
    """tdmd_fast_pipeline_stats -- FastPipelineStats (+ graph / capacity counters)."""
    _fields_ = [("ticks", C.c_int64), ("kernel_launches", C.c_int64), ("rebuilds", C.c_int64),
                ("graph_launches", C.c_int64), ("nlist_retries", C.c_int64),
                ("nlist_capacity", C.c_int64), ("lanes_per_atom", C.c_int32),
                ("nbr_batch", C.c_int32), ("density_lanes_per_atom", C.c_int32),
                ("density_nbr_batch", C.c_int32)]


_p = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_f64 = C.c_double
_pp = C.POINTER(C.c_void_p)
_pi32 = C.POINTER(C.c_int32)
_pf64 = C.POINTER(C.c_double)

# name -> argtypes (all return int32 status unless listed in _RESTYPES)
SIGNATURES = {
    "tdmd_last_error": [],
    "tdmd_abi_version": [],
    "tdmd_copy": [_p, _p, C.c_size_t, _p],
    "tdmd_fast_pipeline_config_default": [C.POINTER(FastPipelineConfig)],
    "tdmd_eam_read_setfl": [C.c_char_p, _pp],
    "tdmd_eam_create": [_i32, _i32, _f64, _i32, _f64, _f64, _p, _p, _p, _pp],
    "tdmd_eam_create_sampled": [_i32, _i32, _f64, _i32, _f64, _f64, _p, _p, _p, _pp],
    "tdmd_eam_destroy": [_p],
    "tdmd_eam_info": [_p, _pi32, _pi32, _pf64, _pi32, _pf64, _pf64],
    "tdmd_set_deterministic_reduce": [_i32],
    "tdmd_get_deterministic_reduce": [_pi32],
    "tdmd_read_lammps_data": [C.c_char_p, _pp],
    "tdmd_system_destroy": [_p],
    "tdmd_system_get": [_p, C.POINTER(_i64), _pi32, _p, _pp, _pp, _pp, _pp, _pp],
    "tdmd_write_lammps_data": [C.c_char_p, C.c_char_p, _i64, _i32, _p, _p, _p, _p, _p, _p],
    "tdmd_read_force_dump": [C.c_char_p, C.POINTER(_i64), _i64, _p, _p, _p, _p],
    "tdmd_write_force_dump": [C.c_char_p, _i64, _i64, _p, _p, _p, _p, _p, _i32],
    "tdmd_write_setfl": [C.c_char_p, _p, C.c_char_p, _p, C.c_char_p],
    "tdmd_eam_coeffs": [_p, _i32, _i32, _p],
    "tdmd_cell_list_create": [_pp],
    "tdmd_cell_list_destroy": [_p],
    "tdmd_cell_list_build": [_p, _p, _i64, C.POINTER(Box), _f64, _p],
    "tdmd_cell_list_get": [_p, _pp, _pp, _pp, _pp, _pi32],
    "tdmd_nlist_create": [_pp],
    "tdmd_nlist_destroy": [_p],
    "tdmd_nlist_build": [_p, _p, _i64, C.POINTER(Box), _f64, _f64, _p],
    "tdmd_nlist_get": [_p, _pp, _pp, _pp, _pi32, C.POINTER(C.c_int64)],
    "tdmd_morse_compute": [_p, _p, _i32, _p, _p, _p, _i32, C.POINTER(Box),
                           C.POINTER(MorseParams), _p, _p, _p],
    "tdmd_morse_compute_zone": [_p, _p, _i32, _p, _p, _p, _i32, _i32, C.POINTER(Box),
                                C.POINTER(MorseParams), _p, _p, _p],
    "tdmd_morse_compute_noalloc": [_p, _p, _i32, _p, _p, _p, _i32, C.POINTER(Box),
                                   C.POINTER(MorseParams), _p, _p, _p],
    "tdmd_device_eam_create": [_p, _pp],
    "tdmd_device_eam_destroy": [_p],
    "tdmd_device_eam_compute": [_p, _p, _p, _i32, _p, _p, _p, _p, _i32, C.POINTER(Box), _p, _p,
                                _p, _p, _p],
    "tdmd_vv_half_kick": [_p, _p, _i32, _p, _p, _i32, _f64, _p],
    "tdmd_vv_drift": [_p, _p, _i32, _f64, C.POINTER(Box), _p],
    "tdmd_vv_fused_kick_drift": [_p, _p, _p, _i32, _p, _p, _i32, _f64, C.POINTER(Box), _i32, _p],
    "tdmd_vv_zero_forces": [_p, _i32, _i32, _p],
    "tdmd_reduce_ke": [_p, _p, _p, _i32, _pf64, _p],
    "tdmd_reduce_vmax": [_p, _i32, _pf64, _p],
    "tdmd_scale_velocities": [_p, _i32, _f64, _p],
    "tdmd_nhc_create": [_f64, _f64, _i32, _f64, _i32, _pp],
    "tdmd_nhc_destroy": [_p],
    "tdmd_nhc_set_t_target": [_p, _f64],
    "tdmd_nhc_half_step": [_p, _f64, _pf64],
    "tdmd_nhc_state": [_p, _p, _p, _p],
    "tdmd_sched_create_morse": [C.POINTER(Box), _i32, C.POINTER(MorseParams),
                                C.POINTER(FastPipelineConfig), _pp],
    "tdmd_sched_create_eam": [C.POINTER(Box), _i32, _p, C.POINTER(FastPipelineConfig), _pp],
    "tdmd_sched_destroy": [_p],
    "tdmd_sched_upload": [_p, _p, _p, _p, _p, _p, _p, _i32],
    "tdmd_sched_run_until": [_p, _i32],
    "tdmd_sched_download": [_p, _p, _p, _p, _p, _p, _i32],
    "tdmd_sched_stats": [_p, C.POINTER(FastPipelineStats)],
    "tdmd_sched_current_step": [_p, _pi32],
    "tdmd_sched_potential_kind": [_p, _pi32],
    "tdmd_sched_interaction_cutoff": [_p, _pf64],
    "tdmd_sched_energies": [_p, _pf64, _pf64, _p],
    "tdmd_sched_energy_log": [_p, _p, _i32, _pi32],
    "tdmd_sched_thermostat_state": [_p, _pf64, _p, _p],
    "tdmd_sched_device_state": [_p, _pp, _pp, _pp],
    "tdmd_sched_atom_order": [_p, _pp],
    "tdmd_sched_neighbor_list": [_p, _p, _p, _i64, _p],
    "tdmd_sched_stream": [_p, _pp],
    "tdmd_batch_create_morse": [_i32, C.POINTER(Box), _p, C.POINTER(MorseParams),
                                C.POINTER(FastPipelineConfig), _pp],
    "tdmd_batch_create_eam": [_i32, C.POINTER(Box), _p, _p, C.POINTER(FastPipelineConfig), _pp],
    "tdmd_batch_destroy": [_p],
    "tdmd_batch_upload": [_p, _p, _p, _p, _p, _i32],
    "tdmd_batch_run_until": [_p, _i32],
    "tdmd_batch_download": [_p, _p, _p, _p],
    "tdmd_batch_energies": [_p, _p, _p],
    "tdmd_batch_energy_log": [_p, _p, _p, _i32, _pi32],
    "tdmd_batch_stats": [_p, C.POINTER(FastPipelineStats)],
    "tdmd_batch_info": [_p, _pi32, C.POINTER(C.c_int64), _pi32, _pi32],
    "tdmd_batch_autotune": [_p, _p, _p, _p],
    "tdmd_batch_last_window_ms": [_p, _pf64],
    "tdmd_batch_stream": [_p, _pp],
    "tdmd_fit_create": [_i32, _i32, C.POINTER(Box), _p, _p, _f64, _i32, _pp],
    "tdmd_fit_destroy": [_p],
    "tdmd_fit_set_targets": [_p, _p],
    "tdmd_fit_morse": [_p, _p, _p, _p, _p, _p],
    "tdmd_fit_eam": [_p, _i32, _i32, _f64, _i32, _f64, _p, _p, _p, _p, _p, _p, _p, _p, _p],
    "tdmd_fit_info": [_p, C.POINTER(C.c_int64), _pi32],
    "tdmd_sched_set_profiling": [_p, _i32],
    "tdmd_sched_autotune": [_p, _p, _p, _p],
    "tdmd_sched_last_window_ms": [_p, _pf64],
    "tdmd_sched_kernel_times": [_p, _p, _p, _i32],
}
_RESTYPES = {"tdmd_last_error": C.c_char_p, "tdmd_abi_version": C.c_int32,
             "tdmd_fast_pipeline_config_default": None}

_lib = None


def lib():
    """The loaded CUDA library (raises when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m tdmd_claude_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, C.c_int32)
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != TDMD_OK:
        msg = lib().tdmd_last_error()
        raise TdmdError(status, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))
