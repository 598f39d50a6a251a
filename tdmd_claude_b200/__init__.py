"""tdmd_claude_b200 -- B200-native (sm_100a) TDMD force + integration path.

A from-scratch CUDA implementation of tdmd_Claude's single-GPU hot path
(cell binning -> Verlet list -> Morse / 3-pass EAM -> velocity-Verlet with an
optional Nose-Hoover chain, FP64 energy/virial reductions) behind the C ABI
in include/tdmd_b200.h.  This package is the Python face of that ABI (see
api.py); the C++ face is include/tdmd_b200.hpp.
"""
from .api import (DeviceCellList, DeviceEam, DeviceNeighborList, EamAlloy,  # noqa: F401
                  FastPipelineScheduler, NoseHooverChain, ReplicaBatch, compute_morse_gpu,
                  compute_morse_gpu_zone, device_compute_ke, device_compute_vmax, device_drift,
                  device_fused_full_kick_drift, device_fused_half_kick_drift, device_half_kick, device_scale_velocities,
                  device_zero_forces, deterministic_reduce, make_config,
                  set_deterministic_reduce)
from ._lib import (TDMD_FP64, TDMD_MIXED, TDMD_POT_EAM, TDMD_POT_MORSE, Box,  # noqa: F401
                   FastPipelineConfig, FastPipelineStats, MorseParams, TdmdError)

__all__ = [
    "Box", "MorseParams", "FastPipelineConfig", "FastPipelineStats", "TdmdError", "EamAlloy",
    "FastPipelineScheduler", "ReplicaBatch", "DeviceNeighborList", "DeviceCellList", "DeviceEam",
    "compute_morse_gpu", "compute_morse_gpu_zone", "device_half_kick", "device_drift",
    "device_fused_half_kick_drift", "device_fused_full_kick_drift", "device_zero_forces",
    "device_compute_ke", "device_compute_vmax", "device_scale_velocities", "NoseHooverChain", "make_config",
    "set_deterministic_reduce", "deterministic_reduce",
    "TDMD_FP64", "TDMD_MIXED", "TDMD_POT_MORSE", "TDMD_POT_EAM",
]
