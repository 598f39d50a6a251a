"""Seeded synthetic inputs of the benchmark and parity configurations.

* fcc_lattice: atoms in the order of tools/gen_fcc_data.py (z, y, x cells,
  then the 4 basis atoms), 1-based ids = index + 1.
* maxwell_boltzmann: init_velocities of benchmarks/phase1_baseline/
  bench_pipeline_scheduler.cu:137-190 -- Gaussian sigma = sqrt(kB T /
  (m mvv2e)), centre-of-mass momentum removed, rescaled to exactly T with
  N_dof = 3N - 3.
* analytic EAM tables (density f, pair phi, embedding F) tabulated on
  setfl grids, smoothly switched to zero over [r_on, r_cut] with the C2
  quintic S(t) = 1 - 10t^3 + 15t^4 - 6t^5, t = (r - r_on)/(r_cut - r_on).

All randomness comes from numpy.random.default_rng(seed).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

KB = 8.617333262e-5      # eV/K, src/core/constants.hpp:15
MVV2E = 1.0364269e-4     # src/core/constants.hpp:28
CU_MASS = 63.546

# Config-0 Morse for Cu (D, alpha, r0).
CU_MORSE = (0.3429, 1.3588, 2.866)


@dataclass
class System:
    positions: np.ndarray      # (n,3) float64
    velocities: np.ndarray     # (n,3) float64
    types: np.ndarray          # (n,) int32, 1-based
    ids: np.ndarray            # (n,) int32
    masses: np.ndarray         # (ntypes+1,) float64, masses[type]
    lo: tuple
    hi: tuple
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.positions.shape[0]


def fcc_lattice(nx: int, ny: int, nz: int, a: float) -> np.ndarray:
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]], np.float64)
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cells = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1).astype(np.float64)
    pos = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3) * a
    return np.ascontiguousarray(pos)


def maxwell_boltzmann(masses_per_atom: np.ndarray, t_target: float, rng) -> np.ndarray:
    n = masses_per_atom.size
    sigma = np.sqrt(KB * t_target / (masses_per_atom * MVV2E))
    v = rng.standard_normal((n, 3)) * sigma[:, None]
    m = masses_per_atom[:, None]
    v -= (m * v).sum(axis=0) / masses_per_atom.sum()
    ke = 0.5 * (masses_per_atom * MVV2E * (v * v).sum(axis=1)).sum()
    n_dof = 3 * n - 3
    t_cur = 2.0 * ke / (n_dof * KB) if n_dof > 0 else 0.0
    if t_cur > 0:
        v *= np.sqrt(t_target / t_cur)
    return np.ascontiguousarray(v)


def fcc_system(ncell: int, a: float, t_target: float, seed: int, jitter: float = 0.01,
               types=None, masses=(CU_MASS,)) -> System:
    """ncell^3 FCC cells, uniform +-jitter per component, MB velocities."""
    rng = np.random.default_rng(seed)
    pos = fcc_lattice(ncell, ncell, ncell, a)
    n = pos.shape[0]
    L = ncell * a
    if jitter > 0:
        pos += rng.uniform(-jitter, jitter, size=pos.shape)
        pos = np.mod(pos, L)  # wrap the few atoms pushed below 0
        pos[pos >= L] -= L
    if types is None:
        types = np.ones(n, np.int32)
    types = np.ascontiguousarray(types, np.int32)
    mass_tab = np.concatenate([[1.0], np.asarray(masses, np.float64)])
    vel = maxwell_boltzmann(mass_tab[types], t_target, rng)
    return System(pos, vel, types, np.arange(1, n + 1, dtype=np.int32), mass_tab, (0.0, 0.0, 0.0),
                  (L, L, L), dict(ncell=ncell, a=a, t=t_target, seed=seed))


# ---------------------------------------------------------------------------
# Analytic EAM tabulated as setfl arrays
# ---------------------------------------------------------------------------
def switch(r, r_on, r_cut):
    t = np.clip((r - r_on) / (r_cut - r_on), 0.0, 1.0)
    return 1.0 - 10.0 * t ** 3 + 15.0 * t ** 4 - 6.0 * t ** 5


@dataclass
class EamTables:
    ntypes: int
    nrho: int
    drho: float
    nr: int
    dr: float
    cutoff: float
    F: np.ndarray      # (ntypes, nrho)
    rho: np.ndarray    # (ntypes, nr)
    rphi: np.ndarray   # (npairs, nr)  r * phi(r), pairs i<=j
    elements: tuple = ("Cu",)
    masses: tuple = (CU_MASS,)


def analytic_eam(beta_f=(5.0,), A_phi=(0.6,), E_F=(1.2,), re=2.556, beta_phi=8.0,
                 r_on=4.5, r_cut=5.0, nr=2000, nrho=2000, rho_max=30.0,
                 elements=("Cu",), masses=(CU_MASS,)) -> EamTables:
    """f_t(r) = exp(-beta_t (r/re - 1)) S(r);  phi_ab(r) = sqrt(A_a A_b)
    exp(-beta_phi (r/re - 1)) S(r);  F_t(rho) = -E_t sqrt(rho)."""
    nt = len(beta_f)
    dr = r_cut / (nr - 1)
    drho = rho_max / (nrho - 1)
    r = np.arange(nr) * dr
    S = switch(r, r_on, r_cut)
    rho_t = np.stack([np.exp(-b * (r / re - 1.0)) * S for b in beta_f])
    rho_grid = np.arange(nrho) * drho
    F_t = np.stack([-e * np.sqrt(rho_grid) for e in E_F])
    rphi = []
    for i in range(nt):
        for j in range(i, nt):
            amp = np.sqrt(A_phi[i] * A_phi[j])
            rphi.append(r * amp * np.exp(-beta_phi * (r / re - 1.0)) * S)
    return EamTables(nt, nrho, drho, nr, dr, r_cut, F_t, rho_t, np.stack(rphi), tuple(elements),
                     tuple(masses))


def cu_eam_tables() -> EamTables:
    """Single-element Cu analytic EAM (the 131,072-atom benchmark)."""
    return analytic_eam()


def ternary_eam_tables() -> EamTables:
    """Equiatomic ternary alloy: re 2.52, beta 4.8/5.0/5.2, pair 0.55/0.60/0.65,
    embedding 1.1/1.2/1.3, masses 58.69/58.93/52.00."""
    return analytic_eam(beta_f=(4.8, 5.0, 5.2), A_phi=(0.55, 0.60, 0.65), E_F=(1.1, 1.2, 1.3),
                        re=2.52, rho_max=30.0, elements=("A", "B", "C"),
                        masses=(58.69, 58.93, 52.00))


# ---------------------------------------------------------------------------
# Named workloads
# ---------------------------------------------------------------------------
def morse_256(seed: int = 1234) -> System:
    """4x4x4 Cu FCC (256 atoms), a = 3.615, +-0.01 A jitter, 300 K."""
    return fcc_system(4, 3.615, 300.0, seed)


def eam_131k(seed: int = 4321) -> System:
    """32x32x32 Cu FCC (131,072 atoms), a = 3.615, +-0.01 A jitter, 300 K."""
    return fcc_system(32, 3.615, 300.0, seed)


def ternary(ncell: int, seed: int = 99, t_target: float = 1000.0) -> System:
    rng = np.random.default_rng(seed + 1)
    n = 4 * ncell ** 3
    types = rng.integers(1, 4, size=n).astype(np.int32)
    return fcc_system(ncell, 3.56, t_target, seed, types=types, masses=(58.69, 58.93, 52.00))


# Morse parameters of the 256-atom Cu case (D eV, alpha 1/A, r0 A, rc A).
MORSE_CU = (0.3429, 1.3588, 2.866, 6.0)


def replica_set(nrep: int = 512, seed: int = 2024, nmin: int = 4, nmax: int = 16,
                tmin: float = 100.0, tmax: float = 1500.0) -> list:
    """Independent Cu FCC Morse systems: replica r has n_r^3 cells with n_r
    uniform in [nmin, nmax] (256 to 16,384 atoms for 4..16), temperature
    uniform in [tmin, tmax] K, its own seeded jitter and velocities."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(nmin, nmax + 1, size=nrep)
    ts = rng.uniform(tmin, tmax, size=nrep)
    return [fcc_system(int(n), 3.615, float(t), seed + 1 + r) for r, (n, t) in
            enumerate(zip(ns, ts))]
