"""File formats around the path: LAMMPS `atomic` data files and setfl.

* write_lammps_data / read_lammps_data follow read_lammps_data
  (src/io/lammps_data_reader.cpp:33-204): header counts and box, Masses,
  Atoms (id type x y z, stored at index id-1), optional Velocities.
* write_setfl writes the DYNAMO setfl layout that EamAlloy::read_setfl
  (src/potentials/eam_alloy.cpp:90-192) reads: 3 comment lines, element
  line, grid line, per element a header + F + rho, then r*phi per pair i<=j.
* write_force_dump writes `dump custom id type x y z fx fy fz`
  (src/drivers/tdmd_main.cpp:65-95).
"""
from __future__ import annotations

import numpy as np

from .workloads import EamTables, System


def write_setfl(path: str, t: EamTables, comment: str = "analytic EAM") -> None:
    with open(path, "w") as f:
        f.write(f"# {comment}\n# generated by tdmd_claude_b200.io.write_setfl\n#\n")
        f.write(f"{t.ntypes} " + " ".join(t.elements) + "\n")
        f.write(f"{t.nrho} {t.drho:.17g} {t.nr} {t.dr:.17g} {t.cutoff:.17g}\n")

        def block(vals):
            for k in range(0, len(vals), 5):
                f.write(" ".join(f"{v:.17g}" for v in vals[k:k + 5]) + "\n")

        for i in range(t.ntypes):
            f.write(f"{i + 1} {t.masses[i]:.6f} 0.0 fcc\n")
            block(t.F[i])
            block(t.rho[i])
        for p in range(t.rphi.shape[0]):
            block(t.rphi[p])


def write_lammps_data(path: str, s: System, title: str = "tdmd_claude_b200 data") -> None:
    ntypes = s.masses.size - 1
    with open(path, "w") as f:
        f.write(f"{title}\n\n{s.n} atoms\n{ntypes} atom types\n\n")
        for a, (lo, hi) in enumerate(zip(s.lo, s.hi)):
            ax = "xyz"[a]
            f.write(f"{lo:.17g} {hi:.17g} {ax}lo {ax}hi\n")
        f.write("\nMasses\n\n")
        for t in range(1, ntypes + 1):
            f.write(f"{t} {s.masses[t]:.17g}\n")
        f.write("\nAtoms # atomic\n\n")
        for i in range(s.n):
            x, y, z = s.positions[i]
            f.write(f"{s.ids[i]} {s.types[i]} {x:.17g} {y:.17g} {z:.17g}\n")
        f.write("\nVelocities\n\n")
        for i in range(s.n):
            vx, vy, vz = s.velocities[i]
            f.write(f"{s.ids[i]} {vx:.17g} {vy:.17g} {vz:.17g}\n")


def read_lammps_data(path: str) -> System:
    with open(path) as f:
        lines = f.read().splitlines()
    natoms = ntypes = 0
    lo = [0.0] * 3
    hi = [0.0] * 3
    k = 1
    while k < len(lines):
        t = lines[k].strip()
        if t in ("Atoms", "Velocities", "Masses") or t.startswith("Atoms "):
            break
        if "atom types" in t:
            ntypes = int(t.split()[0])
        elif "atoms" in t:
            natoms = int(t.split()[0])
        for a, ax in enumerate("xyz"):
            if f"{ax}lo {ax}hi" in t:
                p = t.split()
                lo[a], hi[a] = float(p[0]), float(p[1])
        k += 1
    if natoms <= 0:
        raise ValueError("no atoms in data file")
    pos = np.zeros((natoms, 3))
    vel = np.zeros((natoms, 3))
    types = np.zeros(natoms, np.int32)
    ids = np.zeros(natoms, np.int32)
    masses = np.ones(ntypes + 1)
    while k < len(lines):
        sec = lines[k].split("#")[0].strip()
        k += 1
        if sec not in ("Masses", "Atoms", "Velocities"):
            continue
        count = ntypes if sec == "Masses" else natoms
        got = 0
        while got < count and k < len(lines):
            p = lines[k].split()
            k += 1
            if not p:
                continue
            if sec == "Masses":
                masses[int(p[0])] = float(p[1])
            elif sec == "Atoms":
                i = int(p[0]) - 1
                ids[i], types[i] = int(p[0]), int(p[1])
                pos[i] = [float(p[2]), float(p[3]), float(p[4])]
            else:
                i = int(p[0]) - 1
                vel[i] = [float(p[1]), float(p[2]), float(p[3])]
            got += 1
    return System(pos, vel, types, ids, masses, tuple(lo), tuple(hi))


def write_force_dump(path: str, s: System, forces: np.ndarray, step: int = 0) -> None:
    with open(path, "w") as f:
        f.write(f"ITEM: TIMESTEP\n{step}\nITEM: NUMBER OF ATOMS\n{s.n}\n")
        f.write("ITEM: BOX BOUNDS pp pp pp\n")
        for lo, hi in zip(s.lo, s.hi):
            f.write(f"{lo:.17g} {hi:.17g}\n")
        f.write("ITEM: ATOMS id type x y z fx fy fz\n")
        for i in range(s.n):
            x, y, z = s.positions[i]
            fx, fy, fz = forces[i]
            f.write(f"{s.ids[i]} {s.types[i]} {x:.17g} {y:.17g} {z:.17g} "
                    f"{fx:.17g} {fy:.17g} {fz:.17g}\n")


def read_force_dump(path: str):
    """(ids, types, positions, forces) of a `id type x y z fx fy fz` dump."""
    with open(path) as f:
        lines = f.read().splitlines()
    k = lines.index("ITEM: NUMBER OF ATOMS") + 1
    n = int(lines[k])
    start = next(i for i, l in enumerate(lines) if l.startswith("ITEM: ATOMS")) + 1
    rows = np.array([[float(x) for x in l.split()] for l in lines[start:start + n]])
    order = np.argsort(rows[:, 0])
    rows = rows[order]
    return rows[:, 0].astype(np.int32), rows[:, 1].astype(np.int32), rows[:, 2:5], rows[:, 5:8]
