"""ctypes bindings for the checker libraries built by oracle/Makefile.

Test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg import this module to CHECK or TIME against the reference
algorithm.  The product package (tdmd_claude_b200) never imports it.

* ``liboracle.so``  -- plain-C restatement (tdmd_oracle.c).
* ``_ref/libtdmd_ref.so`` -- the reference's own CPU path compiled from its
  sources (present when the reference tree was available at build time).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(_HERE, "liboracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libtdmd_ref.so")

_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64 = C.c_int64
_i32 = C.c_int32
_f64 = C.c_double


class OrcBox(C.Structure):
    _fields_ = [("lo", C.c_double * 3), ("hi", C.c_double * 3), ("periodic", C.c_int32 * 3)]


def make_box(lo, hi, periodic=(1, 1, 1)) -> OrcBox:
    b = OrcBox()
    for a in range(3):
        b.lo[a] = float(lo[a])
        b.hi[a] = float(hi[a])
        b.periodic[a] = int(periodic[a])
    return b


class OrcPotential(C.Structure):
    _fields_ = [("kind", C.c_int32), ("D", C.c_double), ("alpha", C.c_double),
                ("r0", C.c_double), ("rc", C.c_double), ("eam", C.c_void_p)]


def reference_tree() -> str | None:
    """The reference checkout: $TDMD_REFERENCE_TREE when set, else a
    directory named `reference` beside this repository; None when neither
    holds the reference's `src/` (the tests that need it then skip)."""
    env = os.environ.get("TDMD_REFERENCE_TREE")
    cand = env if env else os.path.join(os.path.dirname(os.path.dirname(_HERE)), "reference")
    return cand if os.path.isdir(os.path.join(cand, "src")) else None


def build(ref: bool | None = None) -> None:
    """Compile liboracle.so (and, when the reference tree exists, _ref/: its
    CPU path for the oracle's pins and the CPU baseline, and its GPU
    scheduler in both precision builds for the same-box comparison)."""
    targets = ["all"]
    ref_tree = reference_tree()
    if ref is None:
        ref = ref_tree is not None
    if ref:
        if ref_tree is None:
            raise RuntimeError("reference tree not found: set TDMD_REFERENCE_TREE")
        targets += ["ref", "refgpu", "dropin", "reftests"]
    args = [f"REF={ref_tree}"] if ref_tree else []
    jobs = str(max(1, min(8, os.cpu_count() or 1)))
    subprocess.run(["make", "-s", "-j", jobs, "-C", _HERE, *args, *targets], check=True)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_ORACLE_SO):
            build(ref=False)
        L = C.CDLL(_ORACLE_SO)
        L.orc_cell_grid.argtypes = [C.POINTER(OrcBox), _f64, _i32p, _f64p]
        L.orc_cell_list_build.argtypes = [_f64p, _i64, C.POINTER(OrcBox), _f64, _i32p, _i32p,
                                          _i32p, _i32p, _i32p]
        L.orc_neighbor_list.argtypes = [_f64p, _i64, C.POINTER(OrcBox), _f64, _f64, _i32, _i32p,
                                        _i32p, _i32p, _i64]
        L.orc_neighbor_list.restype = _i64
        L.orc_needs_rebuild.argtypes = [_f64p, _f64p, _i64, _f64]
        L.orc_needs_rebuild.restype = _i32
        L.orc_morse_forces.argtypes = [_f64p, _i64, C.POINTER(OrcBox), _f64, _f64, _f64, _f64,
                                       _i32p, _i32p, _i32p, _f64p, _f64p]
        L.orc_morse_forces.restype = _f64
        L.orc_spline_build.argtypes = [_f64p, _i32, _f64, _f64p]
        L.orc_spline_eval.argtypes = [_f64p, _i32, _f64, _f64, _f64]
        L.orc_spline_eval.restype = _f64
        L.orc_spline_deriv.argtypes = [_f64p, _i32, _f64, _f64, _f64]
        L.orc_spline_deriv.restype = _f64
        L.orc_eam_create.argtypes = [_i32, _i32, _f64, _i32, _f64, _f64, _f64p, _f64p, _f64p]
        L.orc_eam_create.restype = C.c_void_p
        L.orc_eam_destroy.argtypes = [C.c_void_p]
        L.orc_eam_coeffs.argtypes = [C.c_void_p, _i32, _i32, _f64p]
        L.orc_eam_coeffs.restype = _i32
        L.orc_eam_forces.argtypes = [C.c_void_p, _f64p, _i32p, _i64, C.POINTER(OrcBox), _i32p,
                                     _i32p, _i32p, _f64p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]
        L.orc_eam_forces.restype = _f64
        L.orc_half_kick.argtypes = [_f64p, _f64p, _i32p, _f64p, _i64, _f64]
        L.orc_drift.argtypes = [_f64p, _f64p, _i64, _f64, C.POINTER(OrcBox)]
        L.orc_fused_kick_drift.argtypes = [_f64p, _f64p, _f64p, _i32p, _f64p, _i64, _f64,
                                           C.POINTER(OrcBox), _i32]
        L.orc_kinetic_energy.argtypes = [_f64p, _i32p, _f64p, _i64]
        L.orc_kinetic_energy.restype = _f64
        L.orc_vmax.argtypes = [_f64p, _i64]
        L.orc_vmax.restype = _f64
        L.orc_nhc_init.argtypes = [_f64p, _i32, _f64, _f64, _i32]
        L.orc_nhc_half_step.argtypes = [_f64p, _i32, _f64, _f64, _i32, _f64, _f64]
        L.orc_nhc_half_step.restype = _f64
        L.orc_md_run.argtypes = [C.POINTER(OrcPotential), _f64p, _f64p, _f64p, _i32p, _f64p,
                                 _i64, C.POINTER(OrcBox), _f64, _f64, _i32, _i32p, _i32, _i32,
                                 _f64, _f64, _i32, _f64, _f64, _f64, C.c_void_p, C.c_void_p,
                                 C.c_void_p]
        L.orc_md_run.restype = _i32
        L.orc_morse_fm_loss_grad.argtypes = [_i32, _i64, _f64p, C.POINTER(OrcBox), _f64, _f64,
                                             _f64, _f64, _f64p, _f64p]
        L.orc_morse_fm_loss_grad.restype = _f64
        L.orc_eam_fm_loss_grad.argtypes = [C.c_void_p, _i32, _i64, _f64p, _i32p,
                                           C.POINTER(OrcBox), _f64p, _f64p, _f64p, _f64p]
        L.orc_eam_fm_loss_grad.restype = _f64
        L.orc_eam_set_coeffs.argtypes = [C.c_void_p, _i32, _i32, _f64p]
        L.orc_eam_set_coeffs.restype = _i32
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF_SO)


def ref():
    """The reference's own CPU path (None when it was not built)."""
    global _ref
    if _ref is None:
        if not ref_available():
            return None
        R = C.CDLL(_REF_SO)
        R.ref_last_error.restype = C.c_char_p
        R.ref_read_data.argtypes = [C.c_char_p, C.POINTER(_i64), C.POINTER(_i32), _f64p, _f64p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        R.ref_read_data.restype = _i32
        R.ref_cell_list.argtypes = [_f64p, _i64, _f64p, _f64p, _i32p, _f64, _i32p, C.c_void_p,
                                    C.c_void_p, C.c_void_p]
        R.ref_cell_list.restype = _i32
        R.ref_half_list.argtypes = [_f64p, _i64, _f64p, _f64p, _i32p, _f64, _f64, _i32p, _i32p,
                                    _i32p, _i64]
        R.ref_half_list.restype = _i64
        R.ref_morse_forces.argtypes = [_f64p, _i64, _f64p, _f64p, _i32p, _f64, _f64, _f64, _f64,
                                       _f64, _f64p]
        R.ref_morse_forces.restype = _f64
        R.ref_morse_pair.argtypes = [_f64, _f64, _f64, _f64, _f64, C.POINTER(_f64),
                                     C.POINTER(_f64)]
        R.ref_eam_load.argtypes = [C.c_char_p]
        R.ref_eam_load.restype = C.c_void_p
        R.ref_eam_free.argtypes = [C.c_void_p]
        R.ref_eam_cutoff.argtypes = [C.c_void_p]
        R.ref_eam_cutoff.restype = _f64
        R.ref_eam_ntypes.argtypes = [C.c_void_p]
        R.ref_eam_ntypes.restype = _i32
        R.ref_eam_coeffs.argtypes = [C.c_void_p, _i32, _i32, C.c_void_p]
        R.ref_eam_coeffs.restype = _i32
        R.ref_eam_spline.argtypes = [C.c_void_p, _i32, _i32, _i32, _f64]
        R.ref_eam_spline.restype = _f64
        R.ref_eam_forces.argtypes = [C.c_void_p, _f64p, _i32p, _i64, _f64p, _f64p, _i32p, _f64,
                                     _f64p]
        R.ref_eam_forces.restype = _f64
        R.ref_nhc_create.argtypes = [_f64, _f64, _i32, _f64, _i32]
        R.ref_nhc_create.restype = C.c_void_p
        R.ref_nhc_half_step.argtypes = [C.c_void_p, _f64]
        R.ref_nhc_half_step.restype = _f64
        R.ref_nhc_free.argtypes = [C.c_void_p]
        R.ref_run_cpu.argtypes = [C.c_void_p, _f64, _f64, _f64, _f64, _f64p, _f64p, _f64p, _i32p,
                                  _f64p, _i32, _i64, _f64p, _f64p, _i32p, _f64, _f64, _i32, _i32,
                                  C.POINTER(_f64)]
        R.ref_run_cpu.restype = _f64
        _ref = R
    return _ref


# --------------------------------------------------------------------------
# numpy-level helpers over the C restatement
# --------------------------------------------------------------------------
def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _c32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def cell_list(pos, lo, hi, r_list, periodic=(1, 1, 1)):
    """CellList::build -> (nc, counts, offsets, atoms, atom_cell)."""
    pos = _c64(pos).reshape(-1, 3)
    n = pos.shape[0]
    b = make_box(lo, hi, periodic)
    nc = np.zeros(3, np.int32)
    cs = np.zeros(3, np.float64)
    lib().orc_cell_grid(C.byref(b), r_list, nc, cs)
    ncell = int(nc.prod())
    counts = np.zeros(ncell, np.int32)
    offsets = np.zeros(ncell, np.int32)
    atoms = np.zeros(max(n, 1), np.int32)
    acell = np.zeros(max(n, 1), np.int32)
    lib().orc_cell_list_build(pos.reshape(-1), n, C.byref(b), r_list, nc, counts, offsets, atoms,
                              acell)
    return nc, counts, offsets, atoms[:n], acell[:n]


def neighbor_list(pos, lo, hi, r_cut, r_skin, half, periodic=(1, 1, 1)):
    """Half list (reference CPU) or full list in the reference GPU order.

    Returns (counts, offsets, nbrs) in dense CSR."""
    pos = _c64(pos).reshape(-1, 3)
    n = pos.shape[0]
    b = make_box(lo, hi, periodic)
    counts = np.zeros(max(n, 1), np.int32)
    offsets = np.zeros(max(n, 1), np.int32)
    cap = max(64 * n, 16)
    while True:
        nbrs = np.zeros(cap, np.int32)
        tot = lib().orc_neighbor_list(pos.reshape(-1), n, C.byref(b), r_cut, r_skin,
                                      1 if half else 0, counts, offsets, nbrs, cap)
        if tot <= cap:
            return counts[:n].copy(), offsets[:n].copy(), nbrs[:tot].copy()
        cap = int(tot)


def morse_forces(pos, lo, hi, D, alpha, r0, rc, skin, periodic=(1, 1, 1)):
    """Half-list Morse (compute_pair_forces) -> (pe, forces[n,3], virial6)."""
    pos = _c64(pos).reshape(-1, 3)
    n = pos.shape[0]
    counts, offsets, nbrs = neighbor_list(pos, lo, hi, rc, skin, True, periodic)
    b = make_box(lo, hi, periodic)
    f = np.zeros((n, 3), np.float64)
    w = np.zeros(6, np.float64)
    pe = lib().orc_morse_forces(pos.reshape(-1), n, C.byref(b), D, alpha, r0, rc,
                                _c32(counts), _c32(offsets), _c32(nbrs) if nbrs.size else
                                np.zeros(1, np.int32), f.reshape(-1), w)
    return pe, f, w


def spline_coeffs(values, dr):
    values = _c64(values)
    n = values.size
    coef = np.zeros(4 * (n - 1), np.float64)
    lib().orc_spline_build(values, n, dr, coef)
    return coef


def read_setfl_arrays(path):
    """setfl -> (ntypes, nrho, drho, nr, dr, cutoff, F, rho, rphi), restating
    EamAlloy::read_setfl (eam_alloy.cpp:90-192): 3 comment lines, element
    line, grid line, per element one header line then Nrho + Nr values, then
    Nr values of r*phi per pair i<=j; values may wrap lines freely."""
    with open(path) as f:
        lines = f.read().splitlines()
    if len(lines) < 5:
        raise ValueError("premature end of EAM file")
    ntypes = int(lines[3].split()[0])
    g = lines[4].split()
    nrho, drho, nr, dr, cutoff = int(g[0]), float(g[1]), int(g[2]), float(g[3]), float(g[4])
    k = 5
    pending: list[str] = []

    def take(count):
        nonlocal k, pending
        out = []
        while len(out) < count:
            if not pending:
                if k >= len(lines):
                    raise ValueError("unexpected end of EAM file")
                pending = lines[k].split()
                k += 1
                continue
            out.append(float(pending.pop(0)))
        return out

    F, rho = [], []
    for _ in range(ntypes):
        if pending:          # rest of a value line holds the header
            pending = []
        else:
            while k < len(lines) and not lines[k].strip():
                k += 1
            k += 1           # the element header line
        F.append(take(nrho))
        rho.append(take(nr))
    rphi = [take(nr) for _ in range(ntypes * (ntypes + 1) // 2)]
    return (ntypes, nrho, drho, nr, dr, cutoff, np.array(F), np.array(rho), np.array(rphi))


class OracleEam:
    """EAM tables restated from raw setfl arrays (EamAlloy layout)."""

    @classmethod
    def from_setfl(cls, path):
        return cls(*read_setfl_arrays(path))

    def __init__(self, ntypes, nrho, drho, nr, dr, cutoff, F, rho, rphi):
        self.ntypes, self.nrho, self.drho, self.nr, self.dr, self.cutoff = (
            int(ntypes), int(nrho), float(drho), int(nr), float(dr), float(cutoff))
        self._F, self._rho, self._rphi = _c64(F), _c64(rho), _c64(rphi)
        self.h = lib().orc_eam_create(self.ntypes, self.nrho, self.drho, self.nr, self.dr,
                                      self.cutoff, self._F.reshape(-1), self._rho.reshape(-1),
                                      self._rphi.reshape(-1))

    def __del__(self):
        try:
            lib().orc_eam_destroy(self.h)
        except Exception:
            pass

    def coeffs(self, kind, idx):
        n = self.nrho if kind == 0 else self.nr
        out = np.zeros(4 * (n - 1), np.float64)
        lib().orc_eam_coeffs(self.h, kind, idx, out)
        return out

    def forces(self, pos, types, lo, hi, skin, periodic=(1, 1, 1)):
        """3-pass half-list EAM -> dict(pe, forces, rho, fp, virial, e_embed, e_pair)."""
        pos = _c64(pos).reshape(-1, 3)
        n = pos.shape[0]
        types = _c32(types)
        counts, offsets, nbrs = neighbor_list(pos, lo, hi, self.cutoff, skin, True, periodic)
        b = make_box(lo, hi, periodic)
        f = np.zeros((n, 3), np.float64)
        rho = np.zeros(n, np.float64)
        fp = np.zeros(n, np.float64)
        w = np.zeros(6, np.float64)
        ee = C.c_double(0)
        ep = C.c_double(0)
        nb = _c32(nbrs) if nbrs.size else np.zeros(1, np.int32)
        pe = lib().orc_eam_forces(self.h, pos.reshape(-1), types, n, C.byref(b), _c32(counts),
                                  _c32(offsets), nb, f.reshape(-1), rho.ctypes.data,
                                  fp.ctypes.data, w.ctypes.data, C.addressof(ee),
                                  C.addressof(ep))
        return dict(pe=pe, forces=f, rho=rho, fp=fp, virial=w, e_embed=ee.value,
                    e_pair=ep.value)


    def set_coeffs(self, kind, idx, coef):
        """Overwrites one spline's packed a|b|c|d coefficients."""
        rc = lib().orc_eam_set_coeffs(self.h, kind, idx, _c64(coef))
        assert rc == 0

    def fm_loss_grad(self, pos, types, lo, hi, target, periodic=(1, 1, 1)):
        """Force-matching loss over snapshots pos[s, n, 3] (same box) against
        target[s, n, 3] and its gradient w.r.t. every spline coefficient:
        (loss, gF[nt, 4(nrho-1)], grho[nt, 4(nr-1)], gphi[npairs, 4(nr-1)])."""
        pos = _c64(pos)
        ns, n = pos.shape[0], pos.shape[1]
        types = _c32(np.broadcast_to(np.asarray(types, np.int32).reshape(-1, n), (ns, n)))
        nt = self.ntypes
        gF = np.zeros((nt, 4 * (self.nrho - 1)), np.float64)
        grho = np.zeros((nt, 4 * (self.nr - 1)), np.float64)
        gphi = np.zeros((nt * (nt + 1) // 2, 4 * (self.nr - 1)), np.float64)
        b = make_box(lo, hi, periodic)
        loss = lib().orc_eam_fm_loss_grad(self.h, ns, n, pos.reshape(-1), types.reshape(-1),
                                          C.byref(b), _c64(target).reshape(-1), gF.reshape(-1),
                                          grho.reshape(-1), gphi.reshape(-1))
        return loss, gF, grho, gphi


def morse_fm_loss_grad(pos, lo, hi, D, alpha, r0, rc, target, periodic=(1, 1, 1)):
    """Force-matching loss of Morse (D, alpha, r0) over snapshots pos[s, n, 3]
    against target[s, n, 3] and its gradient (dL/dD, dL/dalpha, dL/dr0)."""
    pos = _c64(pos)
    ns, n = pos.shape[0], pos.shape[1]
    g = np.zeros(3, np.float64)
    b = make_box(lo, hi, periodic)
    loss = lib().orc_morse_fm_loss_grad(ns, n, pos.reshape(-1), C.byref(b), D, alpha, r0, rc,
                                        _c64(target).reshape(-1), g)
    return loss, g


def kinetic_energy(vel, types, masses):
    vel = _c64(vel).reshape(-1, 3)
    return lib().orc_kinetic_energy(vel.reshape(-1), _c32(types), _c64(masses), vel.shape[0])


def md_run(pos, vel, types, masses, lo, hi, dt, skin, rebuild_every, windows, morse=None,
           eam: OracleEam | None = None, nhc=None, adaptive=None, periodic=(1, 1, 1),
           record=False):
    """FastPipelineScheduler::run_until restated on the CPU (FP64).

    morse = (D, alpha, r0, rc); nhc = (t_target, t_period, chain);
    adaptive = (dt_min, dt_max, c2).  Returns dict(pos, vel, forces, pe, ke, dt)."""
    pos = _c64(pos).reshape(-1, 3).copy()
    vel = _c64(vel).reshape(-1, 3).copy()
    n = pos.shape[0]
    forces = np.zeros_like(pos)
    pot = OrcPotential()
    if eam is not None:
        pot.kind = 1
        pot.eam = eam.h
    else:
        pot.kind = 0
        pot.D, pot.alpha, pot.r0, pot.rc = (float(x) for x in morse)
    windows = _c32(windows)
    last = int(windows.max()) if windows.size else 0
    pe = np.zeros(max(last, 1), np.float64)
    ke = np.zeros(max(last, 1), np.float64)
    dts = np.zeros(max(last, 1), np.float64)
    t_target, t_period, chain = nhc if nhc is not None else (0.0, 0.1, 0)
    dt_min, dt_max, c2 = adaptive if adaptive is not None else (0.0, 0.0, 0.0)
    b = make_box(lo, hi, periodic)
    lib().orc_md_run(C.byref(pot), pos.reshape(-1), vel.reshape(-1), forces.reshape(-1),
                     _c32(types), _c64(masses), n, C.byref(b), dt, skin, rebuild_every, windows,
                     windows.size, int(chain), float(t_target), float(t_period),
                     1 if adaptive is not None else 0, float(dt_min), float(dt_max), float(c2),
                     pe.ctypes.data if record else None, ke.ctypes.data if record else None,
                     dts.ctypes.data if record else None)
    return dict(pos=pos, vel=vel, forces=forces, pe=pe[:last], ke=ke[:last], dt=dts[:last])
