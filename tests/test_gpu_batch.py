"""Batched replicas (tdmd_batch_*) through the C ABI.

Each replica follows FastPipelineScheduler's NVE semantics with the same
per-atom arithmetic, so with equal lanes per atom a replica's trajectory is
bit-identical to a single scheduler's on that replica (both precisions);
per-replica energies agree with the scheduler's to 1e-12 relative (only the
summation order differs)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

# (FCC cells per edge, temperature K): 3-cell and wider grids, uneven sizes.
SPECS = [(4, 300.0), (6, 900.0), (5, 1500.0), (7, 100.0), (4, 600.0)]


def _systems(specs, seed=20):
    from tdmd_claude_b200 import workloads as W
    return [W.fcc_system(n, 3.615, t, seed + k) for k, (n, t) in enumerate(specs)]


def _morse():
    from tdmd_claude_b200 import MorseParams
    return MorseParams.make(*golden("ref_morse_256.json")["morse"])


def _batch(systems, precision, lanes=4, use_graphs=True, **kw):
    from tdmd_claude_b200 import Box, ReplicaBatch, make_config
    cfg = make_config(dt=0.001, r_skin=0.3, rebuild_every=10, precision=precision,
                      lanes_per_atom=lanes, use_graphs=use_graphs, **kw)
    b = ReplicaBatch([Box.make(s.lo, s.hi) for s in systems], [s.n for s in systems], _morse(),
                     cfg)
    b.upload(np.concatenate([s.positions for s in systems]),
             np.concatenate([s.velocities for s in systems]),
             np.concatenate([s.types for s in systems]), systems[0].masses)
    return b


def _single(s, precision, lanes=4):
    from tdmd_claude_b200 import Box, FastPipelineScheduler, make_config
    cfg = make_config(dt=0.001, r_skin=0.3, rebuild_every=10, precision=precision,
                      lanes_per_atom=lanes)
    sc = FastPipelineScheduler(Box.make(s.lo, s.hi), s.n, _morse(), cfg)
    sc.upload(s.positions, s.velocities, None, s.types, s.ids, s.masses)
    return sc


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_replicas_equal_single_schedulers(cuda, precision):
    systems = _systems(SPECS)
    b = _batch(systems, precision)
    for target in (10, 25):
        b.run_until(target)
    pos, vel, frc = b.download()
    pe_b, ke_b = b.energies()
    for r, s in enumerate(systems):
        sc = _single(s, precision)
        sc.run_until(10)
        sc.run_until(25)
        st = sc.download()
        assert np.array_equal(b.replica(pos, r), st.positions), r
        assert np.array_equal(b.replica(vel, r), st.velocities), r
        assert np.array_equal(b.replica(frc, r), st.forces), r
        pe, ke, _ = sc.energies()
        assert abs(pe_b[r] - pe) <= 1e-12 * abs(pe), r
        assert abs(ke_b[r] - ke) <= 1e-12 * abs(ke), r
        sc.close()
    info = b.info()
    assert info["step"] == 25 and info["nreplicas"] == len(SPECS)
    st = b.stats()
    assert st.ticks == 25 and st.rebuilds == 3 and st.graph_launches > 0


def test_batch_dense_replica_equals_single_scheduler(cuda):
    """A replica at twice the FCC density (a = 2.87 A, 2 916 atoms, 4 cells
    per axis, ~45 atoms per cell): its list build keeps more candidates per
    warp slab than the slab's index list holds and sweeps all staged
    candidates instead; forces and two steps stay bit-identical to a single
    scheduler's (whose list build takes the cell-pruned path)."""
    from tdmd_claude_b200 import workloads as W
    systems = [W.fcc_system(9, 2.87, 300.0, 61), W.fcc_system(5, 3.615, 300.0, 62)]
    for precision in ("fp64", "mixed"):
        b = _batch(systems, precision)
        b.run_until(0)
        _, _, f0 = b.download()
        b.run_until(2)
        pos, vel, frc = b.download()
        for r, s in enumerate(systems):
            sc = _single(s, precision)
            sc.run_until(0)
            assert np.array_equal(b.replica(f0, r), sc.download().forces), (precision, r)
            sc.run_until(2)
            st = sc.download()
            assert np.array_equal(b.replica(pos, r), st.positions), (precision, r)
            assert np.array_equal(b.replica(vel, r), st.velocities), (precision, r)
            assert np.array_equal(b.replica(frc, r), st.forces), (precision, r)
            sc.close()
        b.close()


def test_batch_graphs_equal_direct_launches(cuda):
    systems = _systems(SPECS[:3], seed=40)
    a = _batch(systems, "mixed", use_graphs=True)
    d = _batch(systems, "mixed", use_graphs=False)
    for t in (10, 20, 37):
        a.run_until(t)
        d.run_until(t)
    pa, va, _ = a.download()
    pd, vd, _ = d.download()
    assert np.array_equal(pa, pd) and np.array_equal(va, vd)
    assert d.stats().graph_launches == 0


def test_batch_empty_replica_and_energy_log(cuda):
    from tdmd_claude_b200 import Box, ReplicaBatch, make_config
    from tdmd_claude_b200 import workloads as W
    s0 = W.fcc_system(4, 3.615, 300.0, 3)
    s1 = W.fcc_system(5, 3.615, 800.0, 4)
    cfg = make_config(dt=0.001, r_skin=0.3, rebuild_every=10, precision="mixed",
                      lanes_per_atom=4, energy_every=10, energy_log_capacity=8)
    boxes = [Box.make(s0.lo, s0.hi), Box.make((0, 0, 0), (20, 20, 20)), Box.make(s1.lo, s1.hi)]
    b = ReplicaBatch(boxes, [s0.n, 0, s1.n], _morse(), cfg)
    b.upload(np.concatenate([s0.positions, s1.positions]),
             np.concatenate([s0.velocities, s1.velocities]),
             np.concatenate([s0.types, s1.types]), s0.masses)
    for t in (10, 20, 30):
        b.run_until(t)
    steps, pk = b.energy_log()
    assert np.array_equal(steps, [10, 20, 30])
    assert pk.shape == (3, 3, 2)
    assert np.all(pk[:, 1, :] == 0.0)          # the empty replica
    pe, ke = b.energies()
    assert np.allclose(pk[-1, :, 0], pe, rtol=0, atol=0)
    assert np.allclose(pk[-1, :, 1], ke, rtol=0, atol=0)
    # the first replica alone gives the same trajectory
    pos, _, _ = b.download()
    sc = _single(s0, "mixed")
    sc.run_until(10)
    sc.run_until(20)
    sc.run_until(30)
    assert np.array_equal(b.replica(pos, 0), sc.download().positions)
    # total energy of each replica stays close (Morse has no shift at rc,
    # so pairs crossing rc move it slightly)
    etot = pk[:, [0, 2], 0] + pk[:, [0, 2], 1]
    assert np.all(np.abs(etot - etot[0]) / np.array([s0.n, s1.n]) < 1e-3)


def test_batch_autotune_keeps_forces(cuda):
    systems = _systems(SPECS[:4], seed=60)
    b = _batch(systems, "mixed", lanes=0)
    b.run_until(0)
    _, _, f0 = b.download()
    shapes, ms = b.autotune()
    lanes, nb = shapes["force"]
    assert shapes["density"] is None  # Morse: one pass
    assert f"force {lanes}x{nb}" in ms and len(ms) == 12 and all(v > 0 for v in ms.values())
    st = b.stats()
    assert (st.lanes_per_atom, st.nbr_batch) == (lanes, nb)
    _, _, f1 = b.download()
    rel = np.sqrt(((f1 - f0) ** 2).sum() / (f0.astype(np.float64) ** 2).sum())
    assert rel < 1e-5


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("ternary", [False, True])
def test_eam_batch_replicas_equal_single_schedulers(cuda, precision, ternary):
    """EAM replicas (shared tables) advance exactly like single EAM
    schedulers (which fuse the next kick into the force pass in mixed NVE,
    bit-identically); per-replica energies match theirs to 1e-12."""
    from tdmd_claude_b200 import Box, EamAlloy, FastPipelineScheduler, ReplicaBatch, make_config
    from tdmd_claude_b200 import workloads as W
    t = W.ternary_eam_tables() if ternary else W.cu_eam_tables()
    eam = EamAlloy.from_tables(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    rng = np.random.default_rng(8)
    systems = []
    for k, (n, temp) in enumerate([(5, 300.0), (4, 900.0), (6, 600.0)]):
        types = rng.integers(1, t.ntypes + 1, size=4 * n ** 3).astype(np.int32)
        systems.append(W.fcc_system(n, 3.615, temp, 70 + k, types=types,
                                    masses=(63.546,) * t.ntypes))
    cfg = dict(dt=0.001, r_skin=0.3, rebuild_every=10, precision=precision, lanes_per_atom=4)
    # energy log at every window end: the window's last force pass writes the
    # per-atom energies, which must equal the separate energy passes
    b = ReplicaBatch([Box.make(s.lo, s.hi) for s in systems], [s.n for s in systems], eam,
                     make_config(**cfg, energy_every=1, energy_log_capacity=4))
    b.upload(np.concatenate([s.positions for s in systems]),
             np.concatenate([s.velocities for s in systems]),
             np.concatenate([s.types for s in systems]), systems[0].masses)
    for target in (10, 23):
        b.run_until(target)
    pos, vel, frc = b.download()
    pe_b, ke_b = b.energies()
    log_steps, pk = b.energy_log()
    assert np.array_equal(log_steps, [10, 23])
    assert np.array_equal(pk[-1, :, 0], pe_b) and np.array_equal(pk[-1, :, 1], ke_b)
    for r, s in enumerate(systems):
        sc = FastPipelineScheduler(Box.make(s.lo, s.hi), s.n, eam, make_config(**cfg))
        sc.upload(s.positions, s.velocities, None, s.types, s.ids, s.masses)
        sc.run_until(10)
        sc.run_until(23)
        st = sc.download()
        assert np.array_equal(b.replica(pos, r), st.positions), r
        assert np.array_equal(b.replica(vel, r), st.velocities), r
        assert np.array_equal(b.replica(frc, r), st.forces), r
        pe, ke, _ = sc.energies()
        assert abs(pe_b[r] - pe) <= 1e-12 * abs(pe), r
        assert abs(ke_b[r] - ke) <= 1e-12 * abs(ke), r
        sc.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_far_atoms_nonperiodic_replica(cuda, precision):
    """A slab replica (z non-periodic, 7 FCC cells across so its grid has 4
    cells per axis and the batch list build takes the warp-slab path) with
    atoms 2 to 4 box lengths outside its z faces, between two periodic
    replicas: the slab's trajectory equals a single scheduler's bit for
    bit (the list build's far records take the exact FP64 test)."""
    from test_gpu_scheduler import _slab_with_far_atoms
    from tdmd_claude_b200 import Box, FastPipelineScheduler, ReplicaBatch, make_config
    from tdmd_claude_b200 import workloads as W
    pos, vel, types, masses, lo, hi = _slab_with_far_atoms(7)
    per = (1, 1, 0)
    a = W.fcc_system(4, 3.615, 300.0, seed=41)
    c = W.fcc_system(5, 3.615, 700.0, seed=42)
    boxes = [Box.make(a.lo, a.hi), Box.make(lo, hi, per), Box.make(c.lo, c.hi)]
    cfg = make_config(dt=0.001, r_skin=0.3, rebuild_every=10, precision=precision,
                      lanes_per_atom=4)
    b = ReplicaBatch(boxes, [a.n, len(pos), c.n], _morse(), cfg)
    b.upload(np.concatenate([a.positions, pos, c.positions]),
             np.concatenate([a.velocities, vel, c.velocities]),
             np.concatenate([a.types, types, c.types]), masses)
    b.run_until(21)
    bp, bv, bf = b.download()
    sc = FastPipelineScheduler(Box.make(lo, hi, per), len(pos), _morse(), cfg)
    sc.upload(pos, vel, None, types, None, masses)
    sc.run_until(21)
    st = sc.download()
    assert np.array_equal(b.replica(bp, 1), st.positions)
    assert np.array_equal(b.replica(bv, 1), st.velocities)
    assert np.array_equal(b.replica(bf, 1), st.forces)
    # the far dimer (the second and third added atoms) interacts
    assert np.abs(st.forces[-4]).max() > 1e-3
    sc.close()
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_lpt_sharded_batches_equal_unsharded(cuda, precision):
    """The replica workload split over two ranks by LPT, run here as two
    batches one after the other on the one GPU: every replica's state and
    logged energies equal the unsharded batch's bit for bit, gathered back
    in replica order (replicas.gather_by_replica)."""
    from tdmd_claude_b200 import workloads as W
    from tdmd_claude_b200.replicas import gather_by_replica, lpt_partition
    systems = W.replica_set(10, seed=13, nmin=4, nmax=6)
    full = _batch(systems, precision, energy_every=10, energy_log_capacity=8)
    full.run_until(20)
    fp, fv, _ = full.download()
    _, fpk = full.energy_log()
    shards = lpt_partition([s.n for s in systems], 2)
    pos_r, pk_r = [], []
    for mine in shards:
        sub = [systems[i] for i in mine]
        b = _batch(sub, precision, energy_every=10, energy_log_capacity=8)
        b.run_until(20)
        p, v, _ = b.download()
        _, pk = b.energy_log()
        pos_r.append([b.replica(p, k) for k in range(len(sub))])
        pk_r.append([pk[:, k, :] for k in range(len(sub))])
        b.close()
    pos_all = gather_by_replica(pos_r[0] + pos_r[1], shards[0] + shards[1], len(systems))
    pk_all = gather_by_replica(pk_r[0] + pk_r[1], shards[0] + shards[1], len(systems))
    for r in range(len(systems)):
        assert np.array_equal(pos_all[r], full.replica(fp, r)), r
        assert np.array_equal(pk_all[r], fpk[:, r, :]), r
    full.close()
