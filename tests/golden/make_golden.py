"""Regenerates the golden fixtures in tests/golden/ from the reference.

Run where the reference tree is available ($TDMD_REFERENCE_TREE, or a
checkout named `reference` beside this repository) after
`make -C oracle all ref`:

    python tests/golden/make_golden.py               # everything
    python tests/golden/make_golden.py --data-files  # the copied inputs only

Sources of truth, all from the reference itself:
  * two_atoms_morse.json   -- VerifyLab analytic values
                              (verifylab/cases/two-atoms-morse/reference/analytic.json)
  * run0_morse_256.json    -- LAMMPS run-0 forces of the 256-atom Cu FCC with
                              Morse rc 6.0 (verifylab/cases/run0-force-match/
                              forces_morse.dump) + the lattice of
                              tests/data/cu_fcc_256.data + the reference CPU
                              path's PE/forces on it
  * run0_eam_256.json      -- same for the Mishin Cu EAM dump (forces_eam.dump)
  * Cu_mishin1.eam.alloy.xz -- the reference's test potential
                              (tests/data/Cu_mishin1.eam.alloy, Mishin et al.
                              PRB 63, 224106 (2001)), xz-compressed byte for
                              byte, so the EAM run-0 tests run where the
                              reference tree is absent
  * 4atoms.data            -- the reference's data-reader test input
                              (tests/data/4atoms.data), byte for byte, for
                              its LammpsDataReader unit test run against this
                              library's reader
  * ref_*.json             -- outputs of the reference's CPU path (compiled
                              from its sources into oracle/_ref/) on the
                              seeded synthetic inputs of tdmd_claude_b200.workloads
"""
from __future__ import annotations

import ctypes as C
import json
import lzma
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from tdmd_claude_b200 import io as TIO  # noqa: E402
from tdmd_claude_b200 import workloads as W  # noqa: E402

REF = O.reference_tree()
if REF is None:
    sys.exit("reference tree not found: set TDMD_REFERENCE_TREE")
PER = np.ones(3, np.int32)


def dump(name, obj):
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(obj, f, indent=None, separators=(",", ":"))
    print("wrote", name)


def arr(a):
    return np.asarray(a).tolist()


def read_data(path):
    R = O.ref()
    n, nt = C.c_int64(), C.c_int32()
    lo, hi = np.zeros(3), np.zeros(3)
    assert R.ref_read_data(path.encode(), C.byref(n), C.byref(nt), lo, hi, None, None, None,
                           None, None) == 0
    N = n.value
    pos, vel = np.zeros((N, 3)), np.zeros((N, 3))
    ty, ids = np.zeros(N, np.int32), np.zeros(N, np.int32)
    m = np.zeros(nt.value + 1)
    R.ref_read_data(path.encode(), C.byref(n), C.byref(nt), lo, hi, pos.ctypes.data,
                    vel.ctypes.data, ty.ctypes.data, ids.ctypes.data, m.ctypes.data)
    return pos, vel, ty, ids, m, lo, hi


def copy_data_files():
    """Reference test inputs that its unit tests read, copied unchanged."""
    for name in ("4atoms.data",):
        with open(os.path.join(REF, "tests/data", name), "rb") as f:
            raw = f.read()
        with open(os.path.join(HERE, name), "wb") as f:
            f.write(raw)
        print("wrote", name)


def main():
    copy_data_files()
    if "--data-files" in sys.argv:
        return
    O.build(ref=True)
    R = O.ref()
    assert R is not None, "reference harness not built"

    # -- two-atom analytic Morse ------------------------------------------
    with open(os.path.join(REF, "verifylab/cases/two-atoms-morse/reference/analytic.json")) as f:
        a = json.load(f)
    dump("two_atoms_morse.json", dict(
        source="verifylab/cases/two-atoms-morse/reference/analytic.json",
        potential=a["potential"], atoms=a["atoms"], step0=a["step0"]))

    # -- run-0 force match (LAMMPS dumps) -----------------------------------
    pos, vel, ty, ids, m, lo, hi = read_data(os.path.join(REF, "tests/data/cu_fcc_256.data"))
    N = pos.shape[0]
    f = np.zeros((N, 3))
    pe = R.ref_morse_forces(pos.reshape(-1), N, lo, hi, PER, 0.3429, 1.3588, 2.866, 6.0, 1.0,
                            f.reshape(-1))
    _, _, _, fl = TIO.read_force_dump(
        os.path.join(REF, "verifylab/cases/run0-force-match/forces_morse.dump"))
    dump("run0_morse_256.json", dict(
        source=["tests/data/cu_fcc_256.data",
                "verifylab/cases/run0-force-match/forces_morse.dump"],
        lo=arr(lo), hi=arr(hi), positions=arr(pos), masses=arr(m),
        morse=[0.3429, 1.3588, 2.866, 6.0], skin=1.0,
        lammps_forces=arr(fl), lammps_pe=-867.64593,
        reference_pe=pe, reference_forces=arr(f),
        tolerance_fp64=1e-12, tolerance_mixed=5e-5))
    mishin = os.path.join(REF, "tests/data/Cu_mishin1.eam.alloy")
    with open(mishin, "rb") as f:
        raw = f.read()
    with open(os.path.join(HERE, "Cu_mishin1.eam.alloy.xz"), "wb") as f:
        f.write(lzma.compress(raw, preset=9 | lzma.PRESET_EXTREME))
    print("wrote Cu_mishin1.eam.alloy.xz")
    h = R.ref_eam_load(mishin.encode())
    fe = np.zeros((N, 3))
    pe_e = R.ref_eam_forces(h, pos.reshape(-1), ty, N, lo, hi, PER, 1.0, fe.reshape(-1))
    _, _, _, fle = TIO.read_force_dump(
        os.path.join(REF, "verifylab/cases/run0-force-match/forces_eam.dump"))
    dump("run0_eam_256.json", dict(
        source=["tests/data/Cu_mishin1.eam.alloy",
                "verifylab/cases/run0-force-match/forces_eam.dump"],
        potential_file="Cu_mishin1.eam.alloy.xz", skin=1.0,
        lammps_forces=arr(fle), lammps_pe=-906.29591, reference_pe=pe_e,
        reference_forces=arr(fe), tolerance_fp64=1e-12, tolerance_mixed=1e-4))
    R.ref_eam_free(h)

    # -- reference CPU path on the synthetic c0 input ----------------------
    s = W.morse_256()
    N = s.n
    lo, hi = np.array(s.lo), np.array(s.hi)
    f = np.zeros((N, 3))
    pe = R.ref_morse_forces(s.positions.reshape(-1), N, lo, hi, PER, 0.3429, 1.3588, 2.866, 6.0,
                            0.3, f.reshape(-1))
    cnt, off = np.zeros(N, np.int32), np.zeros(N, np.int32)
    nb = np.zeros(64 * N, np.int32)
    tot = R.ref_half_list(s.positions.reshape(-1), N, lo, hi, PER, 6.0, 0.3, cnt, off, nb, 64 * N)
    ncl = np.zeros(3, np.int32)
    R.ref_cell_list(s.positions.reshape(-1), N, lo, hi, PER, 6.3, ncl, None, None, None)
    ncell = int(ncl.prod())
    cc, co, ca = np.zeros(ncell, np.int32), np.zeros(ncell, np.int32), np.zeros(N, np.int32)
    R.ref_cell_list(s.positions.reshape(-1), N, lo, hi, PER, 6.3, ncl, cc.ctypes.data,
                    co.ctypes.data, ca.ctypes.data)
    # 100 NVE steps of the reference CPU loop (rebuild every 10).
    p2, v2, f2 = s.positions.copy(), s.velocities.copy(), np.zeros((N, 3))
    pe_end = C.c_double()
    R.ref_run_cpu(None, 0.3429, 1.3588, 2.866, 6.0, p2.reshape(-1), v2.reshape(-1),
                  f2.reshape(-1), s.types, s.masses, 1, N, lo, hi, PER, 0.001, 0.3, 10, 100,
                  C.byref(pe_end))
    dump("ref_morse_256.json", dict(
        workload="tdmd_claude_b200.workloads.morse_256(seed=1234)",
        seed=1234, skin=0.3, morse=[0.3429, 1.3588, 2.866, 6.0],
        positions=arr(s.positions), velocities=arr(s.velocities), masses=arr(s.masses),
        lo=arr(lo), hi=arr(hi), reference_pe=pe, reference_forces=arr(f),
        half_list=dict(total=int(tot), counts=arr(cnt), neighbors=arr(nb[:tot])),
        cell_list=dict(nc=arr(ncl), counts=arr(cc), offsets=arr(co), atoms=arr(ca)),
        md100=dict(dt=0.001, rebuild_every=10, positions=arr(p2), velocities=arr(v2),
                   forces=arr(f2), pe=pe_end.value)))

    # -- reference CPU path on the analytic Cu EAM ---------------------------
    t = W.cu_eam_tables()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "cu_analytic.eam.alloy")
        TIO.write_setfl(path, t)
        h = R.ref_eam_load(path.encode())
        coeffs = {}
        for kind, idx in ((0, 0), (1, 0), (2, 0)):
            nco = R.ref_eam_coeffs(h, kind, idx, None)
            c = np.zeros(nco)
            R.ref_eam_coeffs(h, kind, idx, c.ctypes.data)
            sel = np.linspace(0, nco - 1, 64).astype(int)
            coeffs[f"{kind}_{idx}"] = dict(index=arr(sel), values=arr(c[sel]))
        probes = np.linspace(0.5, 5.2, 40)
        spl = {f"{kind}_{deriv}": [R.ref_eam_spline(h, kind, 0, deriv, float(r)) for r in probes]
               for kind in (1, 2) for deriv in (0, 1)}
        rprobe = np.linspace(0.1, 32.0, 40)
        spl.update({f"0_{deriv}": [R.ref_eam_spline(h, 0, 0, deriv, float(r)) for r in rprobe]
                    for deriv in (0, 1)})
        fe = np.zeros((N, 3))
        pe_e = R.ref_eam_forces(h, s.positions.reshape(-1), s.types, N, lo, hi, PER, 0.3,
                                fe.reshape(-1))
        p2, v2, f2 = s.positions.copy(), s.velocities.copy(), np.zeros((N, 3))
        R.ref_run_cpu(h, 0, 0, 0, 0, p2.reshape(-1), v2.reshape(-1), f2.reshape(-1), s.types,
                      s.masses, 1, N, lo, hi, PER, 0.001, 0.3, 10, 100, C.byref(pe_end))
        R.ref_eam_free(h)
    dump("ref_eam_256.json", dict(
        workload="morse_256(seed=1234) positions with tdmd_claude_b200.workloads.cu_eam_tables()",
        skin=0.3, reference_pe=pe_e, reference_forces=arr(fe), coeffs=coeffs,
        spline_probes=dict(r=arr(probes), rho=arr(rprobe), values=spl),
        md100=dict(dt=0.001, rebuild_every=10, positions=arr(p2), velocities=arr(v2),
                   forces=arr(f2), pe=pe_end.value)))

    # -- NoseHooverChain half steps ------------------------------------------
    seq = []
    for (T, tau, M, dt, ndof) in ((300.0, 0.1, 3, 0.001, 765), (1000.0, 0.05, 1, 0.002, 30),
                                  (500.0, 0.2, 5, 0.001, 3 * 4000 - 3)):
        hh = R.ref_nhc_create(T, tau, M, dt, ndof)
        kes = [12.0 + 3.0 * np.sin(0.1 * k) for k in range(50)]
        if ndof > 1000:
            kes = [0.5 * ndof * 8.617333262e-5 * T * (1.0 + 0.2 * np.cos(0.07 * k)) for k in range(50)]
        scales = [R.ref_nhc_half_step(hh, float(ke)) for ke in kes]
        R.ref_nhc_free(hh)
        seq.append(dict(t_target=T, t_period=tau, chain=M, dt=dt, n_dof=ndof, ke=kes,
                        scale=scales))
    dump("ref_nhc.json", dict(source="NoseHooverChain, src/integrator/device_nose_hoover.cu",
                              cases=seq))


if __name__ == "__main__":
    main()
