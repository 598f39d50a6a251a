"""FastPipelineScheduler on the GPU vs the oracle's restatement of the
reference scheduler loop (oracle.md_run), through the C ABI."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, rel_rms

pytestmark = pytest.mark.gpu


def _wrap_diff(a, b, L):
    d = a - b
    return d - np.round(d / L) * L


def _c0():
    g = golden("ref_morse_256.json")
    return (np.array(g["positions"]), np.array(g["velocities"]), np.array(g["masses"]), g["lo"],
            g["hi"], g["morse"], g["skin"])


def _sched_morse(pos, vel, masses, lo, hi, morse, skin, **cfg):
    from tdmd_claude_b200 import Box, FastPipelineScheduler, MorseParams, make_config
    s = FastPipelineScheduler(Box.make(lo, hi), len(pos), MorseParams.make(*morse),
                              make_config(r_skin=skin, **cfg))
    s.upload(pos, vel, None, np.ones(len(pos), np.int32), None, masses)
    return s


@pytest.mark.parametrize("use_graphs", [True, False])
def test_morse_fp64_trajectory_matches_oracle(cuda, oracle, use_graphs):
    pos, vel, masses, lo, hi, morse, skin = _c0()
    s = _sched_morse(pos, vel, masses, lo, hi, morse, skin, use_graphs=use_graphs)
    windows = [1, 10, 25, 60, 100]
    for w in windows:
        s.run_until(w)
    st = s.download()
    r = oracle.md_run(pos, vel, np.ones(256, np.int32), masses, lo, hi, 0.001, skin, 10, windows,
                      morse=morse)
    L = np.array(hi) - np.array(lo)
    assert np.abs(_wrap_diff(st.positions, r["pos"], L)).max() < 1e-10
    assert np.abs(st.velocities - r["vel"]).max() < 1e-9
    assert rel_rms(st.forces, r["forces"]) < 1e-9
    assert s.current_step() == 100
    # reference md100 (CPU driver loop) stays within rounding of this path
    g = golden("ref_morse_256.json")
    assert np.abs(_wrap_diff(st.positions, np.array(g["md100"]["positions"]), L)).max() < 1e-10


def test_run_until_zero_computes_initial_forces_only(cuda, oracle):
    pos, vel, masses, lo, hi, morse, skin = _c0()
    s = _sched_morse(pos, vel, masses, lo, hi, morse, skin)
    s.run_until(0)
    st = s.download()
    assert np.array_equal(st.positions, pos)
    assert np.array_equal(st.velocities, vel)
    pe, fo, _ = oracle.morse_forces(pos, lo, hi, *morse, skin)
    assert rel_rms(st.forces, fo) < 1e-10
    assert s.stats().rebuilds == 1 and s.current_step() == 0


def test_one_step_windows_equal_unfused_verlet(cuda, oracle):
    """run_until one step at a time == plain half-kick/drift/force/half-kick."""
    pos, vel, masses, lo, hi, morse, skin = _c0()
    s = _sched_morse(pos, vel, masses, lo, hi, morse, skin)
    for k in range(1, 21):
        s.run_until(k)
    st = s.download()
    r = oracle.md_run(pos, vel, np.ones(256, np.int32), masses, lo, hi, 0.001, skin, 10,
                      list(range(1, 21)), morse=morse)
    L = np.array(hi) - np.array(lo)
    assert np.abs(_wrap_diff(st.positions, r["pos"], L)).max() < 1e-11
    assert np.abs(st.velocities - r["vel"]).max() < 1e-10


def test_mixed_morse_cross_precision(cuda, oracle):
    """VerifyLab cross-precision-ab: mixed vs FP64 after 100 steps,
    |dx| < 5e-4 A and |dF| < 2e-2 eV/A."""
    pos, vel, masses, lo, hi, morse, skin = _c0()
    s = _sched_morse(pos, vel, masses, lo, hi, morse, skin, precision="mixed")
    s.run_until(100)
    st = s.download()
    r = oracle.md_run(pos, vel, np.ones(256, np.int32), masses, lo, hi, 0.001, skin, 10, [100],
                      morse=morse)
    L = np.array(hi) - np.array(lo)
    assert np.abs(_wrap_diff(st.positions, r["pos"], L)).max() < 5e-4
    assert np.abs(st.forces - r["forces"]).max() < 2e-2
    assert st.forces.dtype == np.float32


def _eam_setup(precision, ncell=6, **cfg):
    from tdmd_claude_b200 import Box, EamAlloy, FastPipelineScheduler, make_config
    from tdmd_claude_b200 import workloads as W
    t = W.cu_eam_tables()
    sysm = W.fcc_system(ncell, 3.615, 300.0, seed=21)
    eam = EamAlloy.from_tables(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    s = FastPipelineScheduler(Box.make(sysm.lo, sysm.hi), sysm.n, eam,
                              make_config(r_skin=0.3, precision=precision, **cfg))
    s.upload(sysm.positions, sysm.velocities, None, sysm.types, sysm.ids, sysm.masses)
    return s, sysm, t


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_eam_trajectory_matches_oracle(cuda, oracle, precision):
    s, sysm, t = _eam_setup(precision)
    s.run_until(50)
    st = s.download()
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    r = oracle.md_run(sysm.positions, sysm.velocities, sysm.types, sysm.masses, sysm.lo, sysm.hi,
                      0.001, 0.3, 10, [50], eam=oe)
    L = np.array(sysm.hi) - np.array(sysm.lo)
    if precision == "fp64":
        assert np.abs(_wrap_diff(st.positions, r["pos"], L)).max() < 1e-10
        assert rel_rms(st.forces, r["forces"]) < 1e-9
    else:
        assert np.abs(_wrap_diff(st.positions, r["pos"], L)).max() < 5e-4
        assert rel_rms(st.forces, r["forces"]) < 1e-4
        # the force error itself, at the mixed path's own positions
        ro = oe.forces(st.positions, sysm.types, sysm.lo, sysm.hi, 0.3)
        assert rel_rms(st.forces, ro["forces"]) <= 1e-5


def test_eam_mixed_step0_forces_vs_oracle(cuda, oracle):
    """Mixed EAM forces at step 0 within the 1e-5 RMS bound of the FP64 oracle."""
    s, sysm, t = _eam_setup("mixed")
    s.run_until(0)
    st = s.download()
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    r = oe.forces(sysm.positions, sysm.types, sysm.lo, sysm.hi, 0.3)
    assert rel_rms(st.forces, r["forces"]) <= 1e-5


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_energies_and_virial(cuda, oracle, precision):
    s, sysm, t = _eam_setup(precision)
    s.run_until(7)
    pe, ke, w = s.energies()
    st = s.download()
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    r = oe.forces(st.positions, sysm.types, sysm.lo, sysm.hi, 0.3)
    ke_o = oracle.kinetic_energy(st.velocities, sysm.types, sysm.masses)
    tol = 1e-10 if precision == "fp64" else 1e-6
    assert abs(pe - r["pe"]) / abs(r["pe"]) < tol
    assert abs(ke - ke_o) / ke_o < 1e-12
    assert np.abs(w - r["virial"]).max() / np.abs(r["virial"]).max() < tol


def test_nve_energy_log_and_drift(cuda):
    """Device energy log: total energy conserved over 2000 steps (smoothly cut
    EAM), and each record matches an on-demand energy evaluation."""
    s, sysm, t = _eam_setup("fp64", ncell=5, energy_every=10, energy_log_capacity=400)
    s.run_until(2000)
    log = s.energy_log()
    assert log.shape[0] == 200
    assert np.array_equal(log[:, 0], np.arange(10, 2001, 10))
    etot = log[:, 1] + log[:, 2]
    drift = abs(etot[-1] - etot[0]) / sysm.n
    assert drift < 1e-5           # eV/atom over 2 ps
    pe, ke, _ = s.energies()
    assert abs(log[-1, 1] - pe) < 1e-9 * abs(pe)
    assert abs(log[-1, 2] - ke) < 1e-9 * abs(ke)


@pytest.mark.parametrize("precision,per_step", [("fp64", 1e-15), ("mixed", 1e-9)])
def test_adr0007_nve_acceptance_100k(cuda, precision, per_step):
    """DeviceNVEDrift.ADR0007AcceptanceTest100k (tests/unit/test_device_nve_drift.cu:158-257):
    the reference's 256-atom Cu data file (perfect lattice, at rest), Morse
    rc 6.0, skin 1.0, dt 1 fs, rebuild every 10 steps, 100 000 steps; the
    total-energy change per step relative to E0 stays under the reference's
    ADR-0007 targets (tests/support/precision_tolerance.hpp:70-71)."""
    g = golden("run0_morse_256.json")
    pos = np.array(g["positions"])
    s = _sched_morse(pos, np.zeros_like(pos), np.array(g["masses"]), g["lo"], g["hi"],
                     g["morse"], 1.0, dt=0.001, rebuild_every=10, precision=precision)
    s.run_until(0)
    pe0, ke0, _ = s.energies()
    s.run_until(100000)
    pe1, ke1, _ = s.energies()
    e0, e1 = pe0 + ke0, pe1 + ke1
    assert abs((e1 - e0) / e0) / 100000 < per_step
    s.close()


def test_nvt_matches_oracle_composition(cuda, oracle):
    """NHC chain 3, tau 0.1 ps at 600 K on the EAM system: trajectory equals
    the oracle composition of NoseHooverChain + VV (pipeline_scheduler order)."""
    s, sysm, t = _eam_setup("fp64", ncell=4, t_target=600.0, t_period=0.1, nhc_length=3)
    s.run_until(30)
    s.run_until(60)
    st = s.download()
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    r = oracle.md_run(sysm.positions, sysm.velocities, sysm.types, sysm.masses, sysm.lo, sysm.hi,
                      0.001, 0.3, 10, [30, 60], eam=oe, nhc=(600.0, 0.1, 3))
    L = np.array(sysm.hi) - np.array(sysm.lo)
    assert np.abs(_wrap_diff(st.positions, r["pos"], L)).max() < 1e-10
    assert np.abs(st.velocities - r["vel"]).max() < 1e-9


def test_nvt_temperature_control(cuda):
    """test_nvt_thermostat.cu:105-167: <T> within 15 % of the target."""
    from tdmd_claude_b200.workloads import KB
    s, sysm, t = _eam_setup("mixed", ncell=5, t_target=500.0, t_period=0.05, nhc_length=3,
                            energy_every=10, energy_log_capacity=1000)
    s.run_until(4000)
    log = s.energy_log()
    T = 2.0 * log[:, 2] / ((3 * sysm.n - 3) * KB)
    tmean = T[len(T) // 2:].mean()
    assert abs(tmean - 500.0) / 500.0 < 0.15


def test_adaptive_dt_matches_oracle(cuda, oracle):
    pos, vel, masses, lo, hi, morse, skin = _c0()
    s = _sched_morse(pos, vel * 8.0, masses, lo, hi, morse, skin, adaptive_dt=True, dt_min=1e-4,
                     dt_max=0.002, c2=0.05)
    s.run_until(40)
    st = s.download()
    dt, _, _ = s.thermostat_state()
    r = oracle.md_run(pos, vel * 8.0, np.ones(256, np.int32), masses, lo, hi, 0.001, skin, 10,
                      [40], morse=morse, adaptive=(1e-4, 0.002, 0.05), record=True)
    L = np.array(hi) - np.array(lo)
    assert np.abs(_wrap_diff(st.positions, r["pos"], L)).max() < 1e-9
    assert 1e-4 <= dt <= 0.002


def test_kernel_launch_accounting(cuda):
    """Morse NVE, one window without rebuild: 1 (initial force) + 1 window
    prologue (the state copy an overflow retry rewinds to) + 2 per step + 1
    closing half kick, plus the initial list build: 3 kernels (the upload
    already binned the atoms into the cell order, so the cell list is an
    identity fill; then the row-sizing count pass and the fill)."""
    pos, vel, masses, lo, hi, morse, skin = _c0()
    s = _sched_morse(pos, vel, masses, lo, hi, morse, skin, use_graphs=False)
    s.run_until(5)
    st = s.stats()
    assert st.kernel_launches == 3 + 1 + 1 + 2 * 5 + 1
    assert st.ticks == 5 and st.rebuilds == 1


def test_graph_replay_equals_direct_launches(cuda):
    pos, vel, masses, lo, hi, morse, skin = _c0()
    a = _sched_morse(pos, vel, masses, lo, hi, morse, skin, use_graphs=True)
    b = _sched_morse(pos, vel, masses, lo, hi, morse, skin, use_graphs=False)
    for w in (10, 20, 30, 45, 90):
        a.run_until(w)
        b.run_until(w)
    sa, sb = a.download(), b.download()
    assert np.array_equal(sa.positions, sb.positions)
    assert np.array_equal(sa.velocities, sb.velocities)
    assert a.stats().graph_launches > 0 and b.stats().graph_launches == 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("mode", ["nve", "nvt", "nvt_adaptive_dt"])
def test_deterministic_replay(cuda, precision, mode):
    """EamDeterministicReplay (tests/unit/test_fast_pipeline_eam.cu) and
    NVTThermostat.DeterministicReproducibility (test_nvt_thermostat.cu:203-250):
    two runs of the same input are bit-identical, the NHC chain and the
    adaptive dt included."""
    cfg = {"nve": {}, "nvt": dict(t_target=300.0, t_period=0.1, nhc_length=3),
           "nvt_adaptive_dt": dict(t_target=300.0, t_period=0.1, nhc_length=3,
                                   adaptive_dt=True)}[mode]
    s1, _, _ = _eam_setup(precision, ncell=5, **cfg)
    s2, _, _ = _eam_setup(precision, ncell=5, **cfg)
    s1.run_until(100)
    s2.run_until(100)
    a, b = s1.download(), s2.download()
    assert np.array_equal(a.positions, b.positions)
    assert np.array_equal(a.velocities, b.velocities)
    assert np.array_equal(a.forces, b.forces)
    (p1, k1, w1), (p2, k2, w2) = s1.energies(), s2.energies()
    assert p1 == p2 and k1 == k2 and np.array_equal(w1, w2)


def test_neighbor_overflow_retry(cuda, oracle):
    """Squeezing a gas into a dense cluster overflows the padded rows: the
    window is re-run with a larger capacity and still matches the oracle."""
    from tdmd_claude_b200 import Box, FastPipelineScheduler, MorseParams, make_config
    rng = np.random.default_rng(3)
    L = 30.0
    n = 300
    pos = rng.uniform(0, L, size=(n, 3))
    centre = np.array([15.0, 15.0, 15.0])
    vel = (centre - pos) * 1.0           # all atoms drift to the centre
    masses = np.array([1.0, 63.546])
    morse = (0.01, 1.0, 3.0, 5.0)
    s = FastPipelineScheduler(Box.make((0, 0, 0), (L, L, L)), n, MorseParams.make(*morse),
                              make_config(r_skin=1.0, rebuild_every=5, dt=0.002))
    s.upload(pos, vel, None, np.ones(n, np.int32), None, masses)
    s.run_until(200)
    st = s.download()
    assert s.stats().nlist_retries >= 1
    r = oracle.md_run(pos, vel, np.ones(n, np.int32), masses, (0, 0, 0), (L, L, L), 0.002, 1.0, 5,
                      [200], morse=morse)
    assert np.abs(_wrap_diff(st.positions, r["pos"], L)).max() < 1e-8


def test_upload_rejects_bad_types(cuda):
    from tdmd_claude_b200 import TdmdError
    pos, vel, masses, lo, hi, morse, skin = _c0()
    from tdmd_claude_b200 import Box, FastPipelineScheduler, MorseParams, make_config
    s = FastPipelineScheduler(Box.make(lo, hi), 256, MorseParams.make(*morse), make_config())
    bad = np.ones(256, np.int32)
    bad[3] = 7
    with pytest.raises(TdmdError):
        s.upload(pos, vel, None, bad, None, masses)
    with pytest.raises(TdmdError):
        s.run_until(3)     # nothing uploaded


def test_ternary_scheduler_mixed_forces_vs_oracle(cuda, oracle):
    """The scheduler's mixed multi-type path carries each atom's type in the
    low mantissa bits of its F'(rho) gather word: its forces and energy stay
    within the mixed bounds of the FP64 oracle, at the start and after 20
    steps (oracle forces of the scheduler's own positions)."""
    from tdmd_claude_b200 import Box, EamAlloy, FastPipelineScheduler, make_config
    from tdmd_claude_b200 import workloads as W
    t = W.ternary_eam_tables()
    sysm = W.ternary(6, seed=3)
    eam = EamAlloy.from_tables(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    s = FastPipelineScheduler(Box.make(sysm.lo, sysm.hi), sysm.n, eam,
                              make_config(r_skin=0.3, precision="mixed", lanes_per_atom=2))
    s.upload(sysm.positions, sysm.velocities, None, sysm.types, sysm.ids, sysm.masses)
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    for step in (0, 20):
        s.run_until(step)
        st = s.download()
        pe, _, _ = s.energies()
        r = oe.forces(st.positions, sysm.types, sysm.lo, sysm.hi, 0.3)
        assert rel_rms(st.forces, r["forces"]) < 1e-5, step
        assert abs(pe - r["pe"]) / abs(r["pe"]) < 1e-6, step
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("periodic", [(1, 1, 0), (0, 0, 0)])
def test_eam_nonperiodic_matches_oracle(cuda, oracle, precision, periodic):
    """A slab (vacuum along z) and a free cluster: with 8 A of vacuum on
    each non-periodic axis, the neighbor rows take no image across those
    axes and the trajectory follows the oracle's."""
    from tdmd_claude_b200 import Box, EamAlloy, FastPipelineScheduler, make_config
    from tdmd_claude_b200 import workloads as W
    t = W.cu_eam_tables()
    sysm = W.fcc_system(5, 3.615, 300.0, seed=33)
    lo, hi = np.array(sysm.lo, float), np.array(sysm.hi, float)
    for a in range(3):
        if not periodic[a]:
            lo[a] -= 8.0
            hi[a] += 8.0
    eam = EamAlloy.from_tables(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    s = FastPipelineScheduler(Box.make(lo, hi, periodic), sysm.n, eam,
                              make_config(r_skin=0.3, precision=precision, lanes_per_atom=2))
    s.upload(sysm.positions, sysm.velocities, None, sysm.types, sysm.ids, sysm.masses)
    s.run_until(40)
    st = s.download()
    s.close()
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    r = oracle.md_run(sysm.positions, sysm.velocities, sysm.types, sysm.masses, lo, hi, 0.001,
                      0.3, 10, [40], eam=oe, periodic=periodic)
    d = _wrap_diff(st.positions, r["pos"], hi - lo)
    if precision == "fp64":
        assert np.abs(d).max() < 1e-10
        assert rel_rms(st.forces, r["forces"]) < 1e-9
    else:
        assert np.abs(d).max() < 5e-4
        assert rel_rms(st.forces, r["forces"]) < 1e-4


def _slab_with_far_atoms(ncell=5):
    """ncell^3 Cu slab (z non-periodic, 8 A of vacuum) plus atoms far past the
    z faces, where the cell list clamps them into the edge cells: one 2 Lz
    out, a dimer (2.5 A apart) 3.3 Lz out, and one 4 Lz - 1 A above a
    surface atom (a fixed-point frame of width 4 Lz would wrap it onto a
    point 1 A from that atom)."""
    from tdmd_claude_b200 import workloads as W
    sysm = W.fcc_system(ncell, 3.615, 300.0, seed=34)
    lo, hi = np.array(sysm.lo, float), np.array(sysm.hi, float)
    lo[2] -= 8.0
    hi[2] += 8.0
    Lz = hi[2] - lo[2]
    top = int(np.argmax(sysm.positions[:, 2]))
    extra = np.array([[5.0, 6.0, hi[2] + 2.0 * Lz],
                      [9.0, 9.0, hi[2] + 3.3 * Lz],
                      [9.0, 9.0, hi[2] + 3.3 * Lz + 2.5],
                      [sysm.positions[top, 0], sysm.positions[top, 1],
                       sysm.positions[top, 2] + 4.0 * Lz - 1.0],
                      [4.0, 3.0, lo[2] - 2.2 * Lz]])
    pos = np.concatenate([sysm.positions, extra])
    vel = np.concatenate([sysm.velocities, np.zeros_like(extra)])
    types = np.ones(len(pos), np.int32)
    return pos, vel, types, sysm.masses, lo, hi


@pytest.mark.parametrize("ncell", [5, 6])
def test_far_atoms_nonperiodic_lists_bit_exact(cuda, oracle, ncell):
    """Atoms far outside a non-periodic axis: the free-function cell and
    neighbor lists equal the oracle's (neighbor_list.cpp:50-64 takes every
    delta in FP64), including the far dimer's pair and no pair for the atom
    whose wrapped fixed-point position would sit 1 A from a surface atom.
    ncell 5 gives 3-cell periodic axes (minimum image re-applied in FP32),
    6 gives 4 cells (staging with the bounding-box pruning)."""
    from tdmd_claude_b200 import Box, DeviceCellList, DeviceNeighborList
    pos, vel, types, masses, lo, hi = _slab_with_far_atoms(ncell)
    per = (1, 1, 0)
    d = cuda.as_tensor(pos, dtype=cuda.float64, device="cuda")
    box = Box.make(lo, hi, per)
    cl = DeviceCellList()
    cl.build(d, len(pos), box, 5.3)
    nc, atoms, offs, cnts, acell = cl.arrays()
    enc, ecc, eco, eca, eac = oracle.cell_list(pos, lo, hi, 5.3, per)
    assert np.array_equal(cnts, ecc) and np.array_equal(atoms, eca)
    assert np.array_equal(acell, eac)
    nl = DeviceNeighborList()
    nl.build(d, len(pos), box, 5.0, 0.3)
    c, o, nb = nl.host_csr()
    ec, eo, enb = oracle.neighbor_list(pos, lo, hi, 5.0, 0.3, half=False, periodic=per)
    assert np.array_equal(c, ec) and np.array_equal(o, eo) and np.array_equal(nb, enb)
    n0 = len(pos) - 5
    assert c[n0] == 0 and c[n0 + 3] == 0 and c[n0 + 4] == 0
    assert list(nb[o[n0 + 1]:o[n0 + 1] + c[n0 + 1]]) == [n0 + 2]


@pytest.mark.parametrize("ncell", [5, 6])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_far_atoms_nonperiodic_trajectory(cuda, oracle, precision, ncell):
    """The same system through the scheduler: lists bit-exact at step 0 and
    after the rebuilds of steps 11 and 21, forces and a 21-step trajectory
    against the oracle."""
    from tdmd_claude_b200 import Box, EamAlloy, FastPipelineScheduler, make_config
    from tdmd_claude_b200 import workloads as W
    pos, vel, types, masses, lo, hi = _slab_with_far_atoms(ncell)
    per = (1, 1, 0)
    t = W.cu_eam_tables()
    eam = EamAlloy.from_tables(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    s = FastPipelineScheduler(Box.make(lo, hi, per), len(pos), eam,
                              make_config(r_skin=0.3, precision=precision, lanes_per_atom=2))
    s.upload(pos, vel, None, types, None, masses)
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    s.run_until(0)
    c, o, nb = s.neighbor_list()
    ec, eo, enb = oracle.neighbor_list(pos, lo, hi, 5.0, 0.3, half=False, periodic=per)
    assert np.array_equal(c, ec) and np.array_equal(nb, enb)
    r0 = oe.forces(pos, types, lo, hi, 0.3, periodic=per)
    tol = 1e-10 if precision == "fp64" else 1e-5
    assert rel_rms(s.download().forces, r0["forces"]) <= tol
    s.run_until(21)   # the second rebuild follows the drift of step 21
    st = s.download()
    c, o, nb = s.neighbor_list()
    ec, eo, enb = oracle.neighbor_list(st.positions, lo, hi, 5.0, 0.3, half=False, periodic=per)
    assert np.array_equal(c, ec) and np.array_equal(nb, enb)
    r = oracle.md_run(pos, vel, types, masses, lo, hi, 0.001, 0.3, 10, [21], eam=oe,
                      periodic=per)
    d = _wrap_diff(st.positions, r["pos"], hi - lo)
    if precision == "fp64":
        assert np.abs(d).max() < 1e-10
        assert rel_rms(st.forces, r["forces"]) < 1e-9
    else:
        assert np.abs(d).max() < 5e-4
        ro = oe.forces(st.positions, types, lo, hi, 0.3, periodic=per)
        assert rel_rms(st.forces, ro["forces"]) <= 1e-5
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_autotune_keeps_forces(cuda, precision):
    """The autotuner only reorders the per-atom sums: forces stay within
    rounding, the choice is one of the candidates, later steps still match."""
    s, sysm, t = _eam_setup(precision, ncell=8)
    s.run_until(0)
    f0 = s.download().forces.astype(np.float64)
    shapes, ms = s.autotune()
    for p in ("density", "force"):
        lanes, nb = shapes[p]
        assert lanes in (1, 2, 4, 8, 16, 32) and nb in (2, 4)
        assert f"{p} {lanes}x{nb}" in ms
    assert len(ms) == 24 and all(v > 0 for v in ms.values())
    st = s.stats()
    assert (st.density_lanes_per_atom, st.density_nbr_batch) == shapes["density"]
    assert (st.lanes_per_atom, st.nbr_batch) == shapes["force"]
    f1 = s.download().forces.astype(np.float64)
    assert rel_rms(f1, f0) < (1e-13 if precision == "fp64" else 1e-6)
    s.run_until(20)
    assert s.current_step() == 20


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_neighbor_batch_sizes(cuda, precision):
    """Neighbors per lane sweep (2 or 4) only regroups a lane's loads: with
    one lane per atom each lane still visits its row in order, so the two
    sizes give bit-identical trajectories; with four lanes the per-lane sums
    regroup and the forces agree to rounding.  A fixed size limits the
    autotuner's sweep to it."""
    runs = {}
    for lanes in (1, 4):
        for nb in (2, 4):
            s, _, _ = _eam_setup(precision, ncell=6, lanes_per_atom=lanes, nbr_batch=nb)
            s.run_until(0)
            f = s.download().forces.astype(np.float64)
            s.run_until(20)
            st = s.download()
            assert (s.stats().lanes_per_atom, s.stats().nbr_batch) == (lanes, nb)
            runs[lanes, nb] = (f, st.positions, st.velocities)
            s.close()
    for k in range(3):
        assert np.array_equal(runs[1, 2][k], runs[1, 4][k]), k
    assert rel_rms(runs[4, 2][0], runs[4, 4][0]) < (1e-13 if precision == "fp64" else 1e-6)
    s, _, _ = _eam_setup(precision, ncell=6, lanes_per_atom=4, nbr_batch=2)
    s.run_until(0)
    shapes, ms = s.autotune()
    assert shapes["density"][1] == 2 and shapes["force"][1] == 2
    assert sorted(ms) == sorted(f"{p} {1 << k}x2" for p in ("density", "force") for k in range(6))
    s.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("use_graphs", [True, False])
def test_mixed_eam_fused_kick_equals_unfused(cuda, use_graphs, precision):
    """EAM NVE (both precisions) fuses the next step's kick + drift into the
    force pass except on energy-log steps.  Logging every step (nothing
    fused) and logging never (all but window-end steps fused) give
    bit-identical trajectories; a log every 5 steps carries the right step
    numbers."""
    runs = []
    for every in (0, 1, 5):
        s, sysm, _ = _eam_setup(precision, ncell=5, lanes_per_atom=4, use_graphs=use_graphs,
                                energy_every=every, energy_log_capacity=64)
        for t in (7, 20, 33):
            s.run_until(t)
        st = s.download()
        runs.append((st.positions, st.velocities, st.forces))
        if every == 5:
            log = s.energy_log()
            assert np.array_equal(log[:, 0], np.arange(5, 31, 5))
        s.close()
    for k in range(3):
        assert np.array_equal(runs[0][k], runs[1][k])
        assert np.array_equal(runs[0][k], runs[2][k])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_reupload_reuses_or_grows_rows(cuda, precision):
    """A second upload fills the rows into the capacity sized by the first;
    when a row no longer fits (a denser state) it grows and refills.  Forces
    equal those of a fresh scheduler on the same state."""
    s, sysm, _ = _eam_setup(precision, ncell=6, lanes_per_atom=4)
    s.run_until(0)
    cap0 = s.stats().nlist_capacity
    # squeeze the atoms into 75 % of the box: 134 neighbors within r_list
    # on the ideal lattice, past the capacity the first state sized
    lo = np.array(sysm.lo)
    dense = lo + 0.75 * (sysm.positions - lo)
    for pos in (sysm.positions, dense):
        s.upload(pos, sysm.velocities, None, sysm.types, sysm.ids, sysm.masses)
        s.run_until(0)
        fresh, _, _ = _eam_setup(precision, ncell=6, lanes_per_atom=4)
        fresh.upload(pos, sysm.velocities, None, sysm.types, sysm.ids, sysm.masses)
        fresh.run_until(0)
        assert np.array_equal(s.download().forces, fresh.download().forces)
        fresh.close()
    assert s.stats().nlist_capacity > cap0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_reupload_overflow_caught_by_the_window(cuda, precision):
    """After a re-upload the first list's overflow flag is checked by the
    window that follows rather than before it: a denser state that no longer
    fits the rows is caught there, the window is redone with grown rows and
    recomputed initial forces, and the trajectory equals a fresh
    scheduler's bit for bit."""
    s, sysm, _ = _eam_setup(precision, ncell=6, lanes_per_atom=4)
    s.run_until(0)
    cap0 = s.stats().nlist_capacity
    lo = np.array(sysm.lo)
    dense = lo + 0.75 * (sysm.positions - lo)
    s.upload(dense, sysm.velocities, None, sysm.types, sysm.ids, sysm.masses)
    s.run_until(7)
    st = s.stats()
    assert st.nlist_capacity > cap0 and st.nlist_retries >= 1
    fresh, _, _ = _eam_setup(precision, ncell=6, lanes_per_atom=4)
    fresh.upload(dense, sysm.velocities, None, sysm.types, sysm.ids, sysm.masses)
    fresh.run_until(7)
    a, b = s.download(), fresh.download()
    assert np.array_equal(a.positions, b.positions)
    assert np.array_equal(a.velocities, b.velocities)
    assert np.array_equal(a.forces, b.forces)
    fresh.close()
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_arbitrary_atom_order(cuda, oracle, precision):
    """A shuffled upload (held internally in cell order) gives the oracle's
    trajectory for that order atom for atom and downloads in the caller's
    order (cells list their atoms by the caller's index, so every neighbor
    row is the one the caller's order defines)."""
    from tdmd_claude_b200 import Box, EamAlloy, FastPipelineScheduler, make_config
    from tdmd_claude_b200 import workloads as W
    t = W.cu_eam_tables()
    sysm = W.fcc_system(6, 3.615, 300.0, seed=21)
    eam = EamAlloy.from_tables(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    perm = np.random.default_rng(3).permutation(sysm.n)
    pos, vel = sysm.positions[perm], sysm.velocities[perm]
    s = FastPipelineScheduler(Box.make(sysm.lo, sysm.hi), sysm.n, eam,
                              make_config(r_skin=0.3, precision=precision, lanes_per_atom=4))
    s.upload(pos, vel, None, sysm.types[perm], sysm.ids[perm], sysm.masses)
    s.run_until(0)
    st0 = s.download()
    assert np.array_equal(st0.positions, pos) and np.array_equal(st0.ids, sysm.ids[perm])
    s.run_until(30)
    st = s.download()
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    r = oracle.md_run(pos, vel, sysm.types[perm], sysm.masses, sysm.lo, sysm.hi, 0.001, 0.3, 10,
                      [30], eam=oe)
    L = np.array(sysm.hi) - np.array(sysm.lo)
    tol = 1e-10 if precision == "fp64" else 5e-4
    assert np.abs(_wrap_diff(st.positions, r["pos"], L)).max() < tol


def test_launches_without_programmatic_dependent_launch_agree(cuda, tmp_path):
    """TDMD_PDL=0 (read at the library's first launch) turns off the
    programmatic-serialization attribute: a mixed EAM run in a process with
    it off gives the same bits as one with it on."""
    import os
    import subprocess
    import sys
    script = tmp_path / "run.py"
    script.write_text(
        "import sys, numpy as np\n"
        f"sys.path.insert(0, {os.path.dirname(os.path.abspath(__file__))!r})\n"
        f"sys.path.insert(0, {os.path.dirname(os.path.dirname(os.path.abspath(__file__)))!r})\n"
        "from test_gpu_scheduler import _eam_setup\n"
        "s, _, _ = _eam_setup('mixed', ncell=5)\n"
        "s.run_until(37)\n"
        "st = s.download()\n"
        "np.save(sys.argv[1], np.concatenate([st.positions.ravel(), st.velocities.ravel(),\n"
        "                                     st.forces.astype(np.float64).ravel()]))\n")
    out = {}
    for flag in ("0", "1"):
        path = str(tmp_path / f"pdl{flag}.npy")
        env = dict(os.environ, TDMD_PDL=flag)
        r = subprocess.run([sys.executable, str(script), path], capture_output=True, text=True,
                           timeout=600, env=env)
        assert r.returncode == 0, r.stderr
        out[flag] = np.load(path)
    assert np.array_equal(out["0"], out["1"])


@pytest.mark.parametrize("use_graphs", [True, False])
def test_phase_timing_inside_replayed_windows(cuda, use_graphs):
    """Per-phase timing (tdmd_sched_set_profiling): with graphs, the windows
    replay graphs of their own whose event-record nodes bracket each phase;
    every phase of every step is counted, the phases add up to about the
    window, and the trajectory is that of an untimed run bit for bit."""
    # one fixed launch shape (the autotuner's timed choice could differ)
    a, _, _ = _eam_setup("mixed", ncell=10, use_graphs=use_graphs, lanes_per_atom=4)
    b, _, _ = _eam_setup("mixed", ncell=10, use_graphs=use_graphs, lanes_per_atom=4)
    for s in (a, b):
        s.run_until(10)
    a.set_profiling(True)
    win = []
    for w in range(2, 5):
        a.run_until(10 * w)
        win.append(a.last_window_ms())
    kt = a.kernel_times()
    a.set_profiling(False)
    for w in range(2, 5):  # the same windows (a window fuses its inner kicks)
        b.run_until(10 * w)
    assert kt["force"][1] == 30 and kt["density"][1] == 30  # 3 windows x 10 steps
    assert kt["rebuild"][1] == 3
    assert all(ms > 0 for ms, n in kt.values() if n > 0)
    phases = sum(ms * n for ms, n in kt.values())
    assert 0.5 * sum(win) < phases < 1.05 * sum(win)
    sa, sb = a.download(), b.download()
    assert np.array_equal(sa.positions, sb.positions)
    assert np.array_equal(sa.forces, sb.forces)
    # back to the plain graphs: still the same bits
    a.run_until(50)
    b.run_until(50)
    assert np.array_equal(a.download().velocities, b.download().velocities)
