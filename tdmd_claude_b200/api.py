"""Python face of the C ABI, with the reference's class and function names.

Mirrors the drop-in boundary of tdmd_Claude's single-GPU path:
  FastPipelineScheduler   src/scheduler/fast_pipeline_scheduler.cuh:76-192
  DeviceNeighborList      src/neighbors/device_neighbor_list.cuh:20-65
  DeviceCellList          src/domain/device_cell_list.cuh:16
  compute_morse_gpu       src/potentials/device_morse.cuh:37-41
  EamAlloy / DeviceEam    src/potentials/eam_alloy.hpp:47, device_eam.cuh:26
  device_half_kick, device_drift, device_fused_{half,full}_kick_drift,
  device_zero_forces      src/integrator/device_velocity_verlet.cuh:13-59
  NoseHooverChain, device_compute_ke, device_scale_velocities,
  device_compute_vmax     src/integrator/device_nose_hoover.cuh:26-88

Host arrays are numpy; device arrays are torch CUDA tensors (torch is only
the allocator and stream source here).  Errors raise TdmdError, the
counterpart of tdmd::Error.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (TDMD_FP64, TDMD_MIXED, TDMD_POT_EAM, TDMD_POT_MORSE, Box,  # noqa: F401
                   FastPipelineConfig, FastPipelineStats, MorseParams, TdmdError, call, lib)

PRECISIONS = {"fp64": TDMD_FP64, "mixed": TDMD_MIXED}


def _prec(p) -> int:
    if isinstance(p, str):
        return PRECISIONS[p]
    return int(p)


def _ptr(t) -> C.c_void_p:
    """Device (torch) or host (numpy) buffer address; None -> NULL."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return C.c_void_p(t.data_ptr())
    return C.c_void_p(t.ctypes.data)


def _stream(stream) -> C.c_void_p:
    if stream is None:
        return None
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.reshape(shape) if shape is not None else a


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _autotune(fn, handle):
    """Both passes' chosen shapes {"density": (lanes, batch) or None for
    Morse, "force": (lanes, batch)} and the timings {"<pass> <lanes>x<batch>":
    ms} of every shape measured."""
    lanes = np.zeros(2, np.int32)
    batch = np.zeros(2, np.int32)
    ms = np.zeros(24, np.float64)
    call(fn, handle, _ptr(lanes), _ptr(batch), _ptr(ms))
    shapes = {"density": (int(lanes[0]), int(batch[0])) if lanes[0] > 0 else None,
              "force": (int(lanes[1]), int(batch[1]))}
    timings = {f"{p} {1 << k}x{b}": float(ms[12 * j + 6 * i + k])
               for j, p in enumerate(("density", "force")) for i, b in enumerate((2, 4))
               for k in range(6) if ms[12 * j + 6 * i + k] >= 0}
    return shapes, timings


def make_config(dt=0.001, r_skin=1.0, rebuild_every=10, precision="fp64", use_graphs=True,
                lanes_per_atom=0, t_target=0.0, t_period=0.1, nhc_length=3, adaptive_dt=False,
                dt_min=0.0001, dt_max=0.002, c2=0.05, energy_every=0,
                energy_log_capacity=0, nbr_batch=0) -> FastPipelineConfig:
    """FastPipelineConfig{dt, r_skin, rebuild_every} plus this library's knobs."""
    cfg = FastPipelineConfig()
    lib().tdmd_fast_pipeline_config_default(C.byref(cfg))
    cfg.dt, cfg.r_skin, cfg.rebuild_every = float(dt), float(r_skin), int(rebuild_every)
    cfg.precision = _prec(precision)
    cfg.use_graphs = 1 if use_graphs else 0
    cfg.lanes_per_atom = int(lanes_per_atom)
    cfg.t_target, cfg.t_period, cfg.nhc_length = float(t_target), float(t_period), int(nhc_length)
    cfg.adaptive_dt = 1 if adaptive_dt else 0
    cfg.dt_min, cfg.dt_max, cfg.c2 = float(dt_min), float(dt_max), float(c2)
    cfg.energy_every, cfg.energy_log_capacity = int(energy_every), int(energy_log_capacity)
    cfg.nbr_batch = int(nbr_batch)
    return cfg


# ---------------------------------------------------------------------------
# EAM tables
# ---------------------------------------------------------------------------
class EamAlloy:
    """EamAlloy (src/potentials/eam_alloy.hpp:47): setfl tables as splines."""

    def __init__(self, handle=None):
        self._h = handle

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                lib().tdmd_eam_destroy(self._h)
            except Exception:
                pass
            self._h = None

    def read_setfl(self, path: str) -> "EamAlloy":
        h = C.c_void_p()
        call("tdmd_eam_read_setfl", str(path).encode(), C.byref(h))
        if self._h:
            lib().tdmd_eam_destroy(self._h)
        self._h = h
        return self

    @classmethod
    def from_tables(cls, ntypes, nrho, drho, nr, dr, cutoff, F, rho, rphi) -> "EamAlloy":
        F, rho, rphi = _f64(F), _f64(rho), _f64(rphi)
        h = C.c_void_p()
        call("tdmd_eam_create", int(ntypes), int(nrho), float(drho), int(nr), float(dr),
             float(cutoff), _ptr(F), _ptr(rho), _ptr(rphi), C.byref(h))
        return cls(h)

    @classmethod
    def from_samples(cls, ntypes, nrho, drho, nr, dr, cutoff, F, rho, phi) -> "EamAlloy":
        """Tables from phi(r) samples (the reference EamAlloy's SplineTable
        values) instead of the setfl's r*phi(r)."""
        F, rho, phi = _f64(F), _f64(rho), _f64(phi)
        h = C.c_void_p()
        call("tdmd_eam_create_sampled", int(ntypes), int(nrho), float(drho), int(nr), float(dr),
             float(cutoff), _ptr(F), _ptr(rho), _ptr(phi), C.byref(h))
        return cls(h)

    @property
    def handle(self):
        if not self._h:
            raise TdmdError(5, "EamAlloy has no tables (call read_setfl first)")
        return self._h

    def info(self):
        nt, nrho, nr = C.c_int32(), C.c_int32(), C.c_int32()
        drho, dr, rc = C.c_double(), C.c_double(), C.c_double()
        call("tdmd_eam_info", self.handle, C.byref(nt), C.byref(nrho), C.byref(drho), C.byref(nr),
             C.byref(dr), C.byref(rc))
        return dict(ntypes=nt.value, nrho=nrho.value, drho=drho.value, nr=nr.value, dr=dr.value,
                    cutoff=rc.value)

    def cutoff(self) -> float:
        return self.info()["cutoff"]

    def ntypes(self) -> int:
        return self.info()["ntypes"]

    def coeffs(self, kind: int, index: int) -> np.ndarray:
        """Packed a|b|c|d coefficients (kind 0=F, 1=rho, 2=phi)."""
        inf = self.info()
        n = inf["nrho"] if kind == 0 else inf["nr"]
        out = np.zeros(4 * (n - 1), np.float64)
        call("tdmd_eam_coeffs", self.handle, int(kind), int(index), _ptr(out))
        return out


# ---------------------------------------------------------------------------
# Scheduler
# ---------------------------------------------------------------------------
@dataclass
class State:
    positions: np.ndarray
    velocities: np.ndarray
    forces: np.ndarray
    types: np.ndarray
    ids: np.ndarray


class FastPipelineScheduler:
    """FastPipelineScheduler(box, natoms, MorseParams | EamAlloy, cfg)."""

    def __init__(self, box: Box, natoms: int, potential, cfg: FastPipelineConfig | None = None):
        self.box = box
        self.natoms = int(natoms)
        self.cfg = cfg if cfg is not None else make_config()
        self._eam = None
        h = C.c_void_p()
        if isinstance(potential, MorseParams):
            call("tdmd_sched_create_morse", C.byref(box), self.natoms, C.byref(potential),
                 C.byref(self.cfg), C.byref(h))
        elif isinstance(potential, EamAlloy):
            self._eam = potential
            call("tdmd_sched_create_eam", C.byref(box), self.natoms, potential.handle,
                 C.byref(self.cfg), C.byref(h))
        else:
            raise TypeError("potential must be MorseParams or EamAlloy")
        self._h = h
        self.mixed = self.cfg.precision == TDMD_MIXED

    def __del__(self):
        self.close()

    def close(self):
        if getattr(self, "_h", None):
            try:
                lib().tdmd_sched_destroy(self._h)
            except Exception:
                pass
            self._h = None

    def upload(self, positions, velocities, forces=None, types=None, ids=None, masses=None,
               n_types=None):
        n = self.natoms
        pos = _f64(positions).reshape(n, 3)
        vel = _f64(velocities).reshape(n, 3)
        fdt = np.float32 if self.mixed else np.float64
        frc = None if forces is None else np.ascontiguousarray(forces, dtype=fdt).reshape(n, 3)
        typ = _i32(types if types is not None else np.ones(n, np.int32))
        idv = _i32(ids if ids is not None else np.arange(1, n + 1, dtype=np.int32))
        m = _f64(masses)
        nt = int(n_types) if n_types is not None else m.size
        call("tdmd_sched_upload", self._h, _ptr(pos), _ptr(vel), _ptr(frc), _ptr(typ), _ptr(idv),
             _ptr(m), nt)

    def upload_ptrs(self, pos_ptr, vel_ptr, force_ptr, types_ptr, ids_ptr, masses_ptr, n_types):
        """upload() from raw host addresses (pinned buffers, no copies)."""
        call("tdmd_sched_upload", self._h, C.c_void_p(pos_ptr), C.c_void_p(vel_ptr),
             C.c_void_p(force_ptr) if force_ptr else None, C.c_void_p(types_ptr),
             C.c_void_p(ids_ptr) if ids_ptr else None, C.c_void_p(masses_ptr), int(n_types))

    def run_until(self, target_step: int):
        call("tdmd_sched_run_until", self._h, int(target_step))

    def download(self) -> State:
        n = self.natoms
        pos = np.zeros((n, 3), np.float64)
        vel = np.zeros((n, 3), np.float64)
        frc = np.zeros((n, 3), np.float32 if self.mixed else np.float64)
        typ = np.zeros(n, np.int32)
        idv = np.zeros(n, np.int32)
        call("tdmd_sched_download", self._h, _ptr(pos), _ptr(vel), _ptr(frc), _ptr(typ), _ptr(idv),
             n)
        return State(pos, vel, frc, typ, idv)

    def download_ptrs(self, pos_ptr, vel_ptr, force_ptr):
        call("tdmd_sched_download", self._h, C.c_void_p(pos_ptr), C.c_void_p(vel_ptr),
             C.c_void_p(force_ptr) if force_ptr else None, None, None, self.natoms)

    def stats(self) -> FastPipelineStats:
        s = FastPipelineStats()
        call("tdmd_sched_stats", self._h, C.byref(s))
        return s

    def current_step(self) -> int:
        v = C.c_int32()
        call("tdmd_sched_current_step", self._h, C.byref(v))
        return v.value

    def potential_kind(self) -> int:
        v = C.c_int32()
        call("tdmd_sched_potential_kind", self._h, C.byref(v))
        return v.value

    def interaction_cutoff(self) -> float:
        v = C.c_double()
        call("tdmd_sched_interaction_cutoff", self._h, C.byref(v))
        return v.value

    def energies(self):
        """(PE, KE, virial[6]) of the current state, FP64."""
        pe, ke = C.c_double(), C.c_double()
        w = np.zeros(6, np.float64)
        call("tdmd_sched_energies", self._h, C.byref(pe), C.byref(ke), _ptr(w))
        return pe.value, ke.value, w

    def energy_log(self) -> np.ndarray:
        """Records {step, pe, ke, virial[6]} written every energy_every steps."""
        cnt = C.c_int32()
        call("tdmd_sched_energy_log", self._h, None, 0, C.byref(cnt))
        cap = max(min(cnt.value, self.cfg.energy_log_capacity or 1024), 0)
        rec = np.zeros((max(cap, 1), 9), np.float64)
        call("tdmd_sched_energy_log", self._h, _ptr(rec), cap, C.byref(cnt))
        return rec[:cap]

    def thermostat_state(self):
        dt = C.c_double()
        M = max(int(self.cfg.nhc_length), 1)
        eta = np.zeros(M, np.float64)
        eta_v = np.zeros(M, np.float64)
        call("tdmd_sched_thermostat_state", self._h, C.byref(dt), _ptr(eta), _ptr(eta_v))
        return dt.value, eta, eta_v

    def last_window_ms(self) -> float:
        """Device time of the last run_until window (CUDA events, ms)."""
        v = C.c_double()
        call("tdmd_sched_last_window_ms", self._h, C.byref(v))
        return v.value

    def autotune(self):
        """Pick each gather pass's launch shape (lanes per atom, neighbors
        per lane sweep) by timing it; returns (shapes, timings) as
        _autotune describes."""
        return _autotune("tdmd_sched_autotune", self._h)

    def set_profiling(self, on: bool = True):
        call("tdmd_sched_set_profiling", self._h, 1 if on else 0)

    def kernel_times(self):
        """Average ms per launch and launch counts of the phases
        (kick_drift, rebuild, density, force, other) while profiling."""
        ms = np.zeros(5, np.float64)
        cnt = np.zeros(5, np.int64)
        call("tdmd_sched_kernel_times", self._h, _ptr(ms), _ptr(cnt), 5)
        names = ("kick_drift", "rebuild", "density", "force", "other")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(names)}

    def stream(self) -> int:
        s = C.c_void_p()
        call("tdmd_sched_stream", self._h, C.byref(s))
        return s.value or 0

    def neighbor_list(self):
        """(counts, offsets, neighbors) of the scheduler's current list, in
        the caller's atom order (dense CSR on the host)."""
        n = self.natoms
        cnt = np.zeros(n, np.int32)
        tot = C.c_int64()
        call("tdmd_sched_neighbor_list", self._h, _ptr(cnt), None, 0, C.byref(tot))
        nb = np.zeros(max(tot.value, 1), np.int32)
        call("tdmd_sched_neighbor_list", self._h, _ptr(cnt), _ptr(nb), tot.value, C.byref(tot))
        off = np.zeros(n, np.int32)
        off[1:] = np.cumsum(cnt)[:-1]
        return cnt, off, nb[:tot.value]


# ---------------------------------------------------------------------------
# Batched replicas (no reference counterpart; see tdmd_batch_* in the header)
# ---------------------------------------------------------------------------
class ReplicaBatch:
    """Many independent Morse or EAM systems advanced together (NVE).

    boxes: list of Box, natoms: list of int, potential: MorseParams or
    EamAlloy (shared by all replicas).  Arrays passed to upload hold all
    replicas back to back in replica order."""

    def __init__(self, boxes, natoms, params, cfg: FastPipelineConfig | None = None):
        self.nrep = len(boxes)
        self.natoms = np.ascontiguousarray(natoms, dtype=np.int32)
        assert self.natoms.size == self.nrep
        self.total = int(self.natoms.sum())
        self.offsets = np.concatenate([[0], np.cumsum(self.natoms)]).astype(np.int64)
        self.cfg = cfg if cfg is not None else make_config()
        self.mixed = self.cfg.precision == TDMD_MIXED
        barr = (Box * self.nrep)(*boxes)
        h = C.c_void_p()
        self._eam = None
        if isinstance(params, EamAlloy):
            self._eam = params
            call("tdmd_batch_create_eam", self.nrep, barr, _ptr(self.natoms), params.handle,
                 C.byref(self.cfg), C.byref(h))
        else:
            call("tdmd_batch_create_morse", self.nrep, barr, _ptr(self.natoms), C.byref(params),
                 C.byref(self.cfg), C.byref(h))
        self._h = h

    def __del__(self):
        self.close()

    def close(self):
        if getattr(self, "_h", None):
            try:
                lib().tdmd_batch_destroy(self._h)
            except Exception:
                pass
            self._h = None

    def upload(self, positions, velocities, types, masses):
        n = self.total
        pos = _f64(positions).reshape(n, 3)
        vel = _f64(velocities).reshape(n, 3)
        typ = _i32(types)
        m = _f64(masses)
        call("tdmd_batch_upload", self._h, _ptr(pos), _ptr(vel), _ptr(typ), _ptr(m), m.size)

    def run_until(self, target_step: int):
        call("tdmd_batch_run_until", self._h, int(target_step))

    def download(self):
        n = self.total
        pos = np.zeros((n, 3), np.float64)
        vel = np.zeros((n, 3), np.float64)
        frc = np.zeros((n, 3), np.float32 if self.mixed else np.float64)
        call("tdmd_batch_download", self._h, _ptr(pos), _ptr(vel), _ptr(frc))
        return pos, vel, frc

    def replica(self, arr, r):
        return arr[self.offsets[r]:self.offsets[r + 1]]

    def energies(self):
        pe = np.zeros(self.nrep, np.float64)
        ke = np.zeros(self.nrep, np.float64)
        call("tdmd_batch_energies", self._h, _ptr(pe), _ptr(ke))
        return pe, ke

    def energy_log(self):
        """(steps[w], pe_ke[w, nrep, 2]) of the logged windows."""
        cnt = C.c_int32()
        call("tdmd_batch_energy_log", self._h, None, None, 0, C.byref(cnt))
        w = cnt.value
        steps = np.zeros(max(w, 1), np.float64)
        pk = np.zeros((max(w, 1), self.nrep, 2), np.float64)
        call("tdmd_batch_energy_log", self._h, _ptr(steps), _ptr(pk), w, C.byref(cnt))
        return steps[:w], pk[:w]

    def stats(self) -> FastPipelineStats:
        s = FastPipelineStats()
        call("tdmd_batch_stats", self._h, C.byref(s))
        return s

    def current_step(self) -> int:
        return self.info()["step"]

    def info(self):
        nr, lanes, step = C.c_int32(), C.c_int32(), C.c_int32()
        tot = C.c_int64()
        call("tdmd_batch_info", self._h, C.byref(nr), C.byref(tot), C.byref(lanes),
             C.byref(step))
        return {"nreplicas": nr.value, "natoms": tot.value, "lanes_per_atom": lanes.value,
                "step": step.value}

    def autotune(self):
        """As FastPipelineScheduler.autotune, for the whole batch."""
        return _autotune("tdmd_batch_autotune", self._h)

    def last_window_ms(self) -> float:
        v = C.c_double()
        call("tdmd_batch_last_window_ms", self._h, C.byref(v))
        return v.value

    def stream(self) -> int:
        s = C.c_void_p()
        call("tdmd_batch_stream", self._h, C.byref(s))
        return s.value or 0


# ---------------------------------------------------------------------------
# Free functions on device arrays (torch CUDA tensors).
# ---------------------------------------------------------------------------
def _dev_to_numpy(ptr: int, count: int, dtype) -> np.ndarray:
    out = np.zeros(count, dtype)
    if count:
        call("tdmd_copy", _ptr(out), C.c_void_p(ptr), out.nbytes, None)
    return out


class DeviceCellList:
    """DeviceCellList (src/domain/device_cell_list.cuh:16)."""

    def __init__(self):
        h = C.c_void_p()
        call("tdmd_cell_list_create", C.byref(h))
        self._h = h
        self.natoms = 0

    def __del__(self):
        if getattr(self, "_h", None):
            lib().tdmd_cell_list_destroy(self._h)
            self._h = None

    def build(self, d_positions, natoms, box: Box, r_list, stream=None):
        self.natoms = int(natoms)
        call("tdmd_cell_list_build", self._h, _ptr(d_positions), self.natoms, C.byref(box),
             float(r_list), _stream(stream))

    def arrays(self):
        """Host copies: (nc, cell_atoms, cell_offsets, cell_counts, atom_cells)."""
        pa, po, pc, pac = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
        nc = (C.c_int32 * 3)()
        call("tdmd_cell_list_get", self._h, C.byref(pa), C.byref(po), C.byref(pc), C.byref(pac),
             nc)
        ncell = nc[0] * nc[1] * nc[2]
        return (np.array(list(nc), np.int32), _dev_to_numpy(pa.value, self.natoms, np.int32),
                _dev_to_numpy(po.value, ncell, np.int32), _dev_to_numpy(pc.value, ncell, np.int32),
                _dev_to_numpy(pac.value, self.natoms, np.int32))


class DeviceNeighborList:
    """DeviceNeighborList (src/neighbors/device_neighbor_list.cuh:20): full
    list, dense CSR, reference order."""

    def __init__(self):
        h = C.c_void_p()
        call("tdmd_nlist_create", C.byref(h))
        self._h = h
        self.natoms = 0

    def __del__(self):
        if getattr(self, "_h", None):
            lib().tdmd_nlist_destroy(self._h)
            self._h = None

    def build(self, d_positions, natoms, box: Box, r_cut, r_skin, stream=None):
        self.natoms = int(natoms)
        call("tdmd_nlist_build", self._h, _ptr(d_positions), self.natoms, C.byref(box),
             float(r_cut), float(r_skin), _stream(stream))

    def _get(self):
        pn, po, pc = C.c_void_p(), C.c_void_p(), C.c_void_p()
        mx = C.c_int32()
        tot = C.c_int64()
        call("tdmd_nlist_get", self._h, C.byref(pn), C.byref(po), C.byref(pc), C.byref(mx),
             C.byref(tot))
        return pn.value, po.value, pc.value, mx.value, tot.value

    def d_neighbors(self) -> int:
        return self._get()[0]

    def d_offsets(self) -> int:
        return self._get()[1]

    def d_counts(self) -> int:
        return self._get()[2]

    def max_neighbors(self) -> int:
        return self._get()[3]

    def total_pairs(self) -> int:
        return self._get()[4]

    def host_csr(self):
        """(counts, offsets, neighbors) copied to the host."""
        pn, po, pc, _, tot = self._get()
        return (_dev_to_numpy(pc, self.natoms, np.int32), _dev_to_numpy(po, self.natoms, np.int32),
                _dev_to_numpy(pn, tot, np.int32))


def set_deterministic_reduce(on: bool = True) -> None:
    """The ID-ordered energy mode (the reference's TDMD_DETERMINISTIC_REDUCE
    build, src/core/determinism.hpp:20-24), process-wide."""
    call("tdmd_set_deterministic_reduce", 1 if on else 0)


def deterministic_reduce() -> bool:
    v = C.c_int32()
    call("tdmd_get_deterministic_reduce", C.byref(v))
    return bool(v.value)


def compute_morse_gpu(d_positions, d_forces, d_neighbors, d_offsets, d_counts, natoms, box: Box,
                      params: MorseParams, d_energy=None, d_virial=None, precision="fp64",
                      stream=None):
    """compute_morse_gpu (device_morse.cuh:37): forces stored, energy added."""
    call("tdmd_morse_compute", _ptr(d_positions), _ptr(d_forces), _prec(precision),
         C.c_void_p(int(d_neighbors)) if d_neighbors else None, C.c_void_p(int(d_offsets)),
         C.c_void_p(int(d_counts)), int(natoms), C.byref(box), C.byref(params), _ptr(d_energy),
         _ptr(d_virial), _stream(stream))


def compute_morse_gpu_zone(d_positions, d_forces, d_neighbors, d_offsets, d_counts, first_atom,
                           atom_count, box: Box, params: MorseParams, d_energy=None, d_virial=None,
                           precision="fp64", stream=None):
    """compute_morse_gpu_zone (device_morse_zone.cuh:13-23): forces of atoms
    [first_atom, first_atom + atom_count) ADDED to d_forces, energy added."""
    call("tdmd_morse_compute_zone", _ptr(d_positions), _ptr(d_forces), _prec(precision),
         C.c_void_p(int(d_neighbors)) if d_neighbors else None, C.c_void_p(int(d_offsets)),
         C.c_void_p(int(d_counts)), int(first_atom), int(atom_count), C.byref(box),
         C.byref(params), _ptr(d_energy), _ptr(d_virial), _stream(stream))


class DeviceEam:
    """DeviceEam (src/potentials/device_eam.cuh:26)."""

    def __init__(self):
        self._h = None

    def __del__(self):
        if getattr(self, "_h", None):
            lib().tdmd_device_eam_destroy(self._h)
            self._h = None

    def upload_tables(self, eam: EamAlloy):
        h = C.c_void_p()
        call("tdmd_device_eam_create", eam.handle, C.byref(h))
        if self._h:
            lib().tdmd_device_eam_destroy(self._h)
        self._h = h

    def compute(self, d_positions, d_forces, d_types, d_neighbors, d_offsets, d_counts, natoms,
                box: Box, d_energy=None, d_virial=None, d_rho=None, d_fp=None, precision="fp64",
                stream=None):
        call("tdmd_device_eam_compute", self._h, _ptr(d_positions), _ptr(d_forces),
             _prec(precision), _ptr(d_types), C.c_void_p(int(d_neighbors)) if d_neighbors else None,
             C.c_void_p(int(d_offsets)), C.c_void_p(int(d_counts)), int(natoms), C.byref(box),
             _ptr(d_energy), _ptr(d_virial), _ptr(d_rho), _ptr(d_fp), _stream(stream))


def _fprec(d_forces) -> int:
    import torch
    return TDMD_FP64 if d_forces.dtype == torch.float64 else TDMD_MIXED


def device_half_kick(d_vel, d_forces, d_types, d_masses, natoms, dt, stream=None):
    call("tdmd_vv_half_kick", _ptr(d_vel), _ptr(d_forces), _fprec(d_forces), _ptr(d_types),
         _ptr(d_masses), int(natoms), float(dt), _stream(stream))


def device_drift(d_pos, d_vel, natoms, dt, box: Box, stream=None):
    call("tdmd_vv_drift", _ptr(d_pos), _ptr(d_vel), int(natoms), float(dt), C.byref(box),
         _stream(stream))


def device_fused_half_kick_drift(d_vel, d_pos, d_forces, d_types, d_masses, natoms, dt, box,
                                 stream=None):
    call("tdmd_vv_fused_kick_drift", _ptr(d_vel), _ptr(d_pos), _ptr(d_forces), _fprec(d_forces),
         _ptr(d_types), _ptr(d_masses), int(natoms), float(dt), C.byref(box), 0, _stream(stream))


def device_fused_full_kick_drift(d_vel, d_pos, d_forces, d_types, d_masses, natoms, dt, box,
                                 stream=None):
    call("tdmd_vv_fused_kick_drift", _ptr(d_vel), _ptr(d_pos), _ptr(d_forces), _fprec(d_forces),
         _ptr(d_types), _ptr(d_masses), int(natoms), float(dt), C.byref(box), 1, _stream(stream))


def device_zero_forces(d_forces, natoms, stream=None):
    call("tdmd_vv_zero_forces", _ptr(d_forces), _fprec(d_forces), int(natoms), _stream(stream))


def device_compute_ke(d_vel, d_types, d_masses, natoms, stream=None) -> float:
    v = C.c_double()
    call("tdmd_reduce_ke", _ptr(d_vel), _ptr(d_types), _ptr(d_masses), int(natoms), C.byref(v),
         _stream(stream))
    return v.value


def device_compute_vmax(d_vel, natoms, stream=None) -> float:
    v = C.c_double()
    call("tdmd_reduce_vmax", _ptr(d_vel), int(natoms), C.byref(v), _stream(stream))
    return v.value


def device_scale_velocities(d_vel, natoms, factor, stream=None):
    call("tdmd_scale_velocities", _ptr(d_vel), int(natoms), float(factor), _stream(stream))


class NoseHooverChain:
    """NoseHooverChain (device_nose_hoover.cu:187-289), host object."""

    def __init__(self, t_target=300.0, t_period=0.1, chain_length=3, dt=0.001, n_dof=3):
        h = C.c_void_p()
        call("tdmd_nhc_create", float(t_target), float(t_period), int(chain_length), float(dt),
             int(n_dof), C.byref(h))
        self._h = h
        self.M = int(chain_length)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().tdmd_nhc_destroy(self._h)
            self._h = None

    def half_step(self, ke_current: float) -> float:
        s = C.c_double()
        call("tdmd_nhc_half_step", self._h, float(ke_current), C.byref(s))
        return s.value

    def state(self):
        eta, eta_v, eta_m = (np.zeros(max(self.M, 1)) for _ in range(3))
        call("tdmd_nhc_state", self._h, _ptr(eta), _ptr(eta_v), _ptr(eta_m))
        return eta[:self.M], eta_v[:self.M], eta_m[:self.M]
