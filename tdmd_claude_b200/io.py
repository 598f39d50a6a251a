"""File formats around the path, through the library's native readers and
writers (tdmd_read_lammps_data, tdmd_write_lammps_data,
tdmd_read_force_dump, tdmd_write_force_dump, tdmd_write_setfl):

* read_lammps_data / write_lammps_data: LAMMPS `atomic` data files as
  read_lammps_data (src/io/lammps_data_reader.cpp:33-204) reads them --
  header counts and box, Masses, Atoms (id type x y z, stored at index
  id-1), optional Velocities.
* write_setfl: the DYNAMO setfl layout EamAlloy::read_setfl
  (src/potentials/eam_alloy.cpp:90-192) reads.
* write_force_dump / read_force_dump: `dump custom id type x y z fx fy fz`
  (src/drivers/tdmd_main.cpp:65-95, src/io/dump_reader.cpp:15-55).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import TDMD_FP64, TDMD_MIXED, Box, call, lib
from .workloads import EamTables, System


def _cptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def write_setfl(path: str, t: EamTables, comment: str = "analytic EAM") -> None:
    from .api import EamAlloy
    e = EamAlloy.from_tables(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    masses = np.ascontiguousarray(t.masses, np.float64)
    call("tdmd_write_setfl", path.encode(), e.handle, comment.encode(), _cptr(masses),
         " ".join(t.elements).encode())


def write_eam_setfl(path: str, eam, comment: str | None = None) -> None:
    """An EamAlloy's tables (a setfl read keeps its own comment and element
    header lines unless comment is given)."""
    call("tdmd_write_setfl", path.encode(), eam.handle, comment.encode() if comment else None,
         None, None)


def write_lammps_data(path: str, s: System, title: str = "tdmd_claude_b200 data") -> None:
    ntypes = s.masses.size - 1
    pos = np.ascontiguousarray(s.positions, np.float64)
    vel = np.ascontiguousarray(s.velocities, np.float64) if s.velocities is not None else None
    typ = np.ascontiguousarray(s.types, np.int32)
    ids = np.ascontiguousarray(s.ids, np.int32)
    m = np.ascontiguousarray(s.masses, np.float64)
    box = Box.make(s.lo, s.hi)
    call("tdmd_write_lammps_data", path.encode(), title.encode(), int(s.n), int(ntypes),
         C.byref(box), _cptr(pos), _cptr(vel), _cptr(typ), _cptr(ids), _cptr(m))


def read_lammps_data(path: str) -> System:
    h = C.c_void_p()
    call("tdmd_read_lammps_data", path.encode(), C.byref(h))
    try:
        n, nt, box = C.c_int64(), C.c_int32(), Box()
        pp = [C.c_void_p() for _ in range(5)]
        call("tdmd_system_get", h, C.byref(n), C.byref(nt), C.byref(box),
             *[C.byref(p) for p in pp])
        N, T = n.value, nt.value

        def arr(p, count, ct, dtype):
            return np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(count,)).astype(dtype)

        pos = arr(pp[0], 3 * N, C.c_double, np.float64).reshape(N, 3)
        vel = arr(pp[1], 3 * N, C.c_double, np.float64).reshape(N, 3)
        typ = arr(pp[2], N, C.c_int32, np.int32)
        ids = arr(pp[3], N, C.c_int32, np.int32)
        mas = arr(pp[4], T + 1, C.c_double, np.float64)
        return System(pos, vel, typ, ids, mas, tuple(box.lo), tuple(box.hi))
    finally:
        lib().tdmd_system_destroy(h)


def write_force_dump(path: str, s: System, forces: np.ndarray, step: int = 0) -> None:
    f = np.ascontiguousarray(forces)
    prec = TDMD_MIXED if f.dtype == np.float32 else TDMD_FP64
    f = f if prec == TDMD_MIXED else f.astype(np.float64)
    pos = np.ascontiguousarray(s.positions, np.float64)
    typ = np.ascontiguousarray(s.types, np.int32)
    ids = np.ascontiguousarray(s.ids, np.int32)
    box = Box.make(s.lo, s.hi)
    call("tdmd_write_force_dump", path.encode(), int(step), int(s.n), C.byref(box), _cptr(ids),
         _cptr(typ), _cptr(pos), _cptr(f), prec)


def read_force_dump(path: str):
    """(ids, types, positions, forces) of a `id type x y z fx fy fz` dump,
    sorted by id."""
    n = C.c_int64()
    call("tdmd_read_force_dump", path.encode(), C.byref(n), 0, None, None, None, None)
    N = n.value
    ids = np.zeros(N, np.int32)
    typ = np.zeros(N, np.int32)
    pos = np.zeros((N, 3), np.float64)
    frc = np.zeros((N, 3), np.float64)
    call("tdmd_read_force_dump", path.encode(), C.byref(n), N, _cptr(ids), _cptr(typ),
         _cptr(pos), _cptr(frc))
    return ids, typ, pos, frc
