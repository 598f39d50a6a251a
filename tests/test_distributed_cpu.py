"""Host logic of the multi-rank TD zone ring (tdmd_claude_b200/distributed.py)
on the CPU: the zone partition as the reference deals it
(src/domain/zone_partition.cpp:15-200), the exchange plan every rank derives
from it, and the ring exchange itself run as two and three gloo ranks on
127.0.0.1 over CPU tensors (the GPU path sends the same slices with NCCL).
Unmeasured on more than one GPU."""
from __future__ import annotations

import datetime
import json
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tdmd_claude_b200 import Box
from tdmd_claude_b200.distributed import ZonePartition, _side_ghosts, ring_plan


def _part(lx, rc, n_zones, world, r_list):
    p = ZonePartition()
    p.build(Box.make((0.0, 0.0, 0.0), (lx, 10.0, 10.0)), rc, n_zones)
    p.assign_to_ranks(world)
    p.build_zone_neighbors(r_list)
    return p


def test_partition_follows_reference():
    # n = max(3, floor(L_x / rc)); zone_of truncates and clamps
    p = _part(115.68, 5.0, 0, 1, 5.3)
    assert p.n_zones == 23 and abs(p.width - 115.68 / 23) < 1e-15
    assert list(p.zone_of([-1.0, 0.0, 5.0296, 115.68, 200.0])) == [0, 0, 1, 22, 22]
    assert _part(14.46, 6.0, 0, 1, 7.0).n_zones == 3
    with pytest.raises(ValueError):
        _part(14.46, 6.0, 2, 1, 7.0)
    # ranks get contiguous blocks, the first n % P ranks one zone more
    p = _part(70.0, 10.0, 7, 3, 10.0)
    assert [z.owner_rank for z in p.zones] == [0, 0, 0, 1, 1, 2, 2]
    assert (p.first_zone_of_rank(1), p.n_zones_of_rank(1)) == (3, 2)
    assert p.zone_neighbors(0) == [0, 1, 6] and p.span(10.0) == 1
    assert p.ghost_zones(0) == [3, 6] and p.ghost_zones(1) == [2, 5]
    with pytest.raises(ValueError):
        _part(70.0, 10.0, 3, 4, 10.0)  # fewer zones than ranks
    # assign_atoms: counting sort by zone, input order inside a zone
    x = np.array([65.0, 1.0, 35.0, 2.0, 69.9, 11.0])
    perm = p.assign_atoms(x)
    assert list(perm) == [1, 3, 5, 2, 0, 4]
    assert [(z.atom_offset, z.natoms_in_zone) for z in p.zones] == \
        [(0, 2), (2, 1), (3, 0), (3, 1), (4, 0), (4, 0), (4, 2)]


@pytest.mark.parametrize("nz,world,span", [(3, 2, 2), (4, 2, 1), (7, 3, 1), (7, 3, 2),
                                           (10, 4, 2), (23, 8, 2), (12, 2, 3), (6, 3, 2)])
def test_ring_plan_covers_every_ghost_once(nz, world, span):
    width = 10.0
    p = _part(nz * width, width, nz, world, span * width - 1e-9)
    assert p.span(span * width - 1e-9) == span
    plans = [ring_plan(p, r, world, span) for r in range(world)]
    for r, pl in enumerate(plans):
        got = [z for za, zb in pl.from_prev + pl.from_next for z in range(za, zb)]
        assert sorted(set(got)) == p.ghost_zones(r)
        for za, zb in pl.from_prev:
            assert all(p.owner_rank(z) == pl.prev for z in range(za, zb))
        for za, zb in pl.from_next:
            assert all(p.owner_rank(z) == pl.next for z in range(za, zb))
        # what r sends equals what its neighbors expect, run for run
        assert pl.to_next == plans[pl.next].from_prev
        assert pl.to_prev == plans[pl.prev].from_next
        for za, zb in pl.to_next + pl.to_prev:
            assert all(p.is_local(z, r) for z in range(za, zb))


def test_ring_plan_rejects_ghosts_beyond_the_ring_neighbors():
    p = _part(100.0, 10.0, 10, 4, 25.0)  # span 3 with ranks of 2-3 zones
    with pytest.raises(ValueError, match="ring neighbors"):
        ring_plan(p, 0, 4, 3)
    # one rank: no exchange at all
    q = ring_plan(_part(100.0, 10.0, 10, 1, 25.0), 0, 1, 3)
    assert q.to_next == q.from_prev == []


def test_side_ghosts_are_the_partition_ghosts():
    p = _part(230.0, 10.0, 23, 5, 19.0)
    for r in range(5):
        lo, hi = _side_ghosts(p, r, 2)
        assert sorted(set(lo + hi)) == p.ghost_zones(r)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_main(rank, world, port, nz, span, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from tdmd_claude_b200.distributed import ring_exchange
    p = _part(nz * 10.0, 10.0, nz, world, span * 10.0 - 1e-9)
    rng = np.random.default_rng(3)
    x = rng.uniform(0.0, nz * 10.0, 400)
    p.assign_atoms(x)
    plan = ring_plan(p, rank, world, span)
    # rows of local zones carry (zone, rank, atom); all others NaN
    arr = torch.full((400, 3), float("nan"), dtype=torch.float64)
    for z in range(*plan.local):
        zn = p.zones[z]
        for k in range(zn.atom_offset, zn.atom_offset + zn.natoms_in_zone):
            arr[k] = torch.tensor([z, rank, k], dtype=torch.float64)
    ts = ring_exchange(dist, None, arr, p, plan, 7 + rank)
    res = {"ts": list(ts), "rows": {}}
    for z in range(nz):
        zn = p.zones[z]
        rows = arr[zn.atom_offset:zn.atom_offset + zn.natoms_in_zone]
        res["rows"][z] = rows.tolist()
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump(res, f)


@pytest.mark.parametrize("nz,world,span", [(5, 2, 1), (3, 2, 2), (9, 3, 2)])
def test_ring_exchange_over_gloo(tmp_path, nz, world, span):
    mp.spawn(_exchange_main, args=(world, _free_port(), nz, span, str(tmp_path)), nprocs=world,
             join=True)
    p = _part(nz * 10.0, 10.0, nz, world, span * 10.0 - 1e-9)
    p.assign_atoms(np.random.default_rng(3).uniform(0.0, nz * 10.0, 400))
    for r in range(world):
        res = json.load(open(tmp_path / f"r{r}.json"))
        # time steps reported by the previous and the next rank
        assert res["ts"] == [7 + (r - 1) % world, 7 + (r + 1) % world]
        ghosts = set(p.ghost_zones(r))
        for z in range(nz):
            rows = np.array(res["rows"][str(z)]).reshape(-1, 3)
            if p.is_local(z, r) or z in ghosts:
                own = p.owner_rank(z)
                a = p.zones[z].atom_offset
                want = np.array([[z, own, a + k] for k in range(len(rows))], np.float64)
                assert np.array_equal(rows, want), (r, z)
            else:
                assert np.isnan(rows).all(), (r, z)
