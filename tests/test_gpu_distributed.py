"""The multi-rank TD zone ring (tdmd_claude_b200/distributed.py) and its zone
force call on the GPU.

* compute_morse_gpu_zone (tdmd_morse_compute_zone) over the zones of a system
  equals the whole-system Morse call; it adds to the forces it is given.
* One rank (no process group) against the oracle's scheduler loop
  (oracle.md_run): the reference's 256-atom Morse case, NVE and NVT.
* Two and three ranks as processes sharing this one GPU over gloo (each
  process advances its own zones with the library's kernels; the boundary
  zones go through host tensors; no kernel waits on another process): the
  final state equals the one-rank run bit for bit, FP64 and mixed, NVE and
  NVT, with zones re-assigned at rebuilds on the way.  NCCL's direct device
  exchange needs one GPU per rank and is unmeasured here."""
from __future__ import annotations

import datetime
import os
import socket

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


def _by_id(pos, vel, frc, ids):
    o = np.argsort(ids)
    return pos[o], vel[o], frc[o]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_zone_force_call_equals_whole_system(cuda, oracle, precision):
    torch = cuda
    from tdmd_claude_b200 import (Box, DeviceNeighborList, MorseParams, compute_morse_gpu,
                                  compute_morse_gpu_zone)
    from tdmd_claude_b200 import workloads as W
    s = W.fcc_system(8, 3.615, 600.0, seed=11)
    box = Box.make(s.lo, s.hi)
    mp_ = MorseParams.make(0.3429, 1.3588, 2.866, 6.0)
    d_pos = torch.from_numpy(s.positions).cuda()
    nl = DeviceNeighborList()
    nl.build(d_pos, s.n, box, 6.0, 0.3)
    dt = torch.float64 if precision == "fp64" else torch.float32
    full = torch.zeros((s.n, 3), dtype=dt, device="cuda")
    e_full = torch.zeros(1, dtype=torch.float64, device="cuda")
    compute_morse_gpu(d_pos, full, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), s.n, box, mp_,
                      d_energy=e_full, precision=precision)
    zone = torch.zeros_like(full)
    e_zone = torch.zeros(1, dtype=torch.float64, device="cuda")
    cuts = [0, 700, 701, 1500, s.n]  # ragged ranges, one of a single atom
    for a, b in zip(cuts[:-1], cuts[1:]):
        compute_morse_gpu_zone(d_pos, zone, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), a,
                               b - a, box, mp_, d_energy=e_zone, precision=precision)
    tol = 1e-12 if precision == "fp64" else 1e-6
    assert rel_rms(zone.cpu().numpy(), full.cpu().numpy()) < tol
    assert abs(e_zone.item() - e_full.item()) < tol * abs(e_full.item())
    # forces are ADDED: a second call on one range doubles it, bit for bit
    before = zone.clone()
    compute_morse_gpu_zone(d_pos, zone, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), 701,
                           799, box, mp_, precision=precision)
    assert torch.equal(zone[701:1500], 2 * before[701:1500])
    assert torch.equal(zone[:701], before[:701]) and torch.equal(zone[1500:], before[1500:])
    # an empty range is a no-op; a negative one is an error
    compute_morse_gpu_zone(d_pos, zone, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), 5, 0,
                           box, mp_, precision=precision)
    from tdmd_claude_b200 import TdmdError
    with pytest.raises(TdmdError):
        compute_morse_gpu_zone(d_pos, zone, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), -1,
                               4, box, mp_, precision=precision)


def _one_rank(pos, vel, masses, lo, hi, morse, skin, steps, precision="fp64", **cfg):
    from tdmd_claude_b200 import Box, MorseParams
    from tdmd_claude_b200.distributed import DistributedConfig, DistributedPipelineScheduler
    c = DistributedConfig(dt=0.001, r_skin=skin, rebuild_every=10, precision=precision, **cfg)
    s = DistributedPipelineScheduler(Box.make(lo, hi), len(pos), MorseParams.make(*morse), c)
    s.upload(pos, vel, None, np.ones(len(pos), np.int32), None, masses)
    s.run_until(steps)
    return s


def test_one_rank_matches_oracle_nve(cuda, oracle):
    pos, vel, masses, lo, hi, morse, skin = _c0()
    s = _one_rank(pos, vel, masses, lo, hi, morse, skin, 100)
    p, v, f, t, ids = s.download()
    p, v, f = _by_id(p, v, f, ids)
    r = oracle.md_run(pos, vel, np.ones(256, np.int32), masses, lo, hi, 0.001, skin, 10, [100],
                      morse=morse)
    L = np.array(hi) - np.array(lo)
    assert np.abs(_wrap_diff(p, r["pos"], L)).max() < 1e-10
    assert np.abs(v - r["vel"]).max() < 1e-9
    assert rel_rms(f, r["forces"]) < 1e-9
    # zone bookkeeping: 3 zones on one rank, every zone at step 100
    part = s.partition()
    assert part.n_zones == 3 and s.rank() == 0 and s.size() == 1
    assert all(z.time_step == 100 for z in part.zones)
    assert s.min_local_time_step() == s.min_global_time_step() == 100
    st = s.stats()
    assert st.ticks == 100 and st.kernel_launches == 300 and st.exchanges == 0
    assert st.dep_check_calls == 300 and st.dep_check_failures == 0
    # energies: the oracle's at the final state
    pe, ke = s.energies()
    pe_o, _, _ = oracle.morse_forces(r["pos"], lo, hi, *morse, skin)
    assert abs(pe - pe_o) < 1e-10 * abs(pe_o)


def test_one_rank_matches_oracle_nvt(cuda, oracle):
    pos, vel, masses, lo, hi, morse, skin = _c0()
    s = _one_rank(pos, vel, masses, lo, hi, morse, skin, 60, t_target=500.0, t_period=0.1,
                  nhc_length=3)
    p, v, f, t, ids = s.download()
    p, v, f = _by_id(p, v, f, ids)
    r = oracle.md_run(pos, vel, np.ones(256, np.int32), masses, lo, hi, 0.001, skin, 10, [60],
                      morse=morse, nhc=(500.0, 0.1, 3))
    L = np.array(hi) - np.array(lo)
    assert np.abs(_wrap_diff(p, r["pos"], L)).max() < 1e-10
    assert np.abs(v - r["vel"]).max() < 1e-9


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _system(ncell, temp, seed, vac=0.0):
    """ncell^3 FCC Cu; vac > 0 lengthens the box along x by that much
    vacuum (a periodic slab)."""
    from tdmd_claude_b200 import workloads as W
    s = W.fcc_system(ncell, 3.615, temp, seed=seed)
    hi = (s.hi[0] + vac, s.hi[1], s.hi[2])
    return s.positions, s.velocities, s.masses, s.lo, hi


MORSE = (0.3429, 1.3588, 2.866, 6.0)


def _run(world, rank, case, out):
    import torch
    from tdmd_claude_b200 import Box, MorseParams
    from tdmd_claude_b200.distributed import DistributedConfig, DistributedPipelineScheduler
    ncell, temp, precision, nvt, steps, vac = case
    pos, vel, masses, lo, hi = _system(ncell, temp, 5, vac)
    cfg = DistributedConfig(dt=0.001, r_skin=0.3, rebuild_every=10, precision=precision,
                            t_target=temp if nvt else 0.0)
    s = DistributedPipelineScheduler(Box.make(lo, hi), len(pos), MorseParams.make(*MORSE), cfg)
    s.upload(pos, vel, None, np.ones(len(pos), np.int32), None, masses)
    s.run_until(steps // 2)
    s.run_until(steps)
    p, v, f, t, ids = s.download()
    pe, ke = s.energies()
    st = s.stats()
    res = dict(pos=p, vel=v, frc=f, ids=ids, pe=pe, ke=ke, rezones=st.rezones,
               exchanges=st.exchanges, ticks=st.ticks, mgts=s.min_global_time_step(),
               fails=st.dep_check_failures)
    if out is not None:
        np.savez(out, **res)
    torch.cuda.synchronize()
    return res


def _rank_main(rank, world, port, cases, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        for k, case in enumerate(cases):
            _run(world, rank, case, os.path.join(out, f"c{k}_r{rank}.npz"))
        dist.barrier()
    finally:
        dist.destroy_process_group()


CASES = [
    # ncell, T, precision, NVT, steps, vacuum along x
    (8, 900.0, "fp64", False, 60, 0.0),
    (8, 900.0, "mixed", False, 60, 0.0),
    (8, 600.0, "fp64", True, 40, 0.0),
    (6, 900.0, "fp64", False, 30, 0.0),   # 3 zones: the reference test's layout
    # a slab: 8 zones of 6.26 A, the last three empty -- with 3 ranks the
    # last rank owns no atom and sends and receives empty runs
    (8, 900.0, "fp64", False, 30, 21.16),
]


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_give_the_one_rank_bits(cuda, tmp_path, world):
    """Every case of CASES (FP64 / mixed NVE, FP64 NVT, a 3-zone system, a
    slab with empty zones) run by `world` processes: each rank's final state
    is the one-rank state."""
    import torch.multiprocessing as mp
    from tdmd_claude_b200 import Box
    from tdmd_claude_b200.distributed import ZonePartition
    mp.spawn(_rank_main, args=(world, _free_port(), CASES, str(tmp_path)), nprocs=world,
             join=True)
    for k, case in enumerate(CASES):
        pos, _, _, lo, hi = _system(case[0], case[1], 5, case[5])
        zp = ZonePartition()
        zp.build(Box.make(lo, hi), MORSE[3])
        assert zp.n_zones >= world
        one = _run(1, 0, case, None)
        for r in range(world):
            got = np.load(tmp_path / f"c{k}_r{r}.npz")
            for key in ("pos", "vel", "frc", "ids"):
                assert np.array_equal(got[key], one[key]), (case, r, key)
            assert got["pe"] == one["pe"] and got["ke"] == one["ke"]
            assert int(got["exchanges"]) == case[4] and int(got["ticks"]) == case[4]
            assert int(got["mgts"]) == case[4] and int(got["fails"]) == 0
            assert int(got["rezones"]) == one["rezones"]
        if case[0] == 8 and case[5] == 0.0:
            assert one["rezones"] > 0  # atoms crossed zone slabs: zones re-assigned
        if case[5] > 0.0:
            counts = np.bincount(zp.zone_of(pos[:, 0]), minlength=zp.n_zones)
            assert zp.n_zones == 8 and (counts[5:] == 0).all() and (counts[:5] > 0).all()


def _reference_tests_main(rank, world, port, out):
    """The reference's distributed unit tests (tests/unit/
    test_distributed_pipeline.cu:163-390) on its 256-atom Morse fixture,
    skin 1.0: NVE drift over 1000 steps, zone time steps after
    run_until(10), and NVT from 100 K to a 500 K target over 2000 steps."""
    import json

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=300))
    try:
        from tdmd_claude_b200 import Box, MorseParams
        from tdmd_claude_b200 import workloads as W
        from tdmd_claude_b200.distributed import DistributedConfig, DistributedPipelineScheduler
        pos, vel, masses, lo, hi, morse, _ = _c0()
        box, mp_, n = Box.make(lo, hi), MorseParams.make(*morse), len(pos)
        types = np.ones(n, np.int32)
        res = {}
        s = DistributedPipelineScheduler(box, n, mp_, DistributedConfig(r_skin=1.0))
        s.upload(pos, vel, None, types, None, masses)
        s.run_until(10)
        z0, z1 = s.plan.local
        res["zone_steps"] = [s.partition().zones[z].time_step for z in range(z0, z1)]
        res["min_local"] = s.min_local_time_step()
        s.run_until(1)  # already past: no-op
        e0 = sum(s.energies())
        s2 = DistributedPipelineScheduler(box, n, mp_, DistributedConfig(r_skin=1.0))
        s2.upload(pos, vel, None, types, None, masses)
        s2.run_until(1)
        e1 = sum(s2.energies())
        s2.run_until(1000)
        ef = sum(s2.energies())
        res["nve_drift"] = abs((ef - e1) / e1)
        res["e10"] = e0
        v100 = W.maxwell_boltzmann(masses[types], 100.0, np.random.default_rng(42))
        s3 = DistributedPipelineScheduler(box, n, mp_, DistributedConfig(
            r_skin=1.0, t_target=500.0, t_period=0.1, nhc_length=3))
        s3.upload(pos, v100, None, types, None, masses)
        s3.run_until(1000)
        temps = []
        for step in range(1100, 2001, 100):
            s3.run_until(step)
            _, ke = s3.energies()
            temps.append(2.0 * ke / ((3 * n - 3) * W.KB))
        res["t_mean"] = float(np.mean(temps))
        with open(os.path.join(out, f"r{rank}.json"), "w") as f:
            json.dump(res, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_reference_distributed_unit_tests_on_two_ranks(cuda, tmp_path):
    import json

    import torch.multiprocessing as mp
    mp.spawn(_reference_tests_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        res = json.load(open(tmp_path / f"r{r}.json"))
        assert res["min_local"] >= 10 and all(t >= 10 for t in res["zone_steps"])
        assert res["nve_drift"] < 1e-4
        assert abs(res["t_mean"] - 500.0) / 500.0 < 0.30
