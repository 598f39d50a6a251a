"""Multi-rank TD zone ring: the reference's DistributedPipelineScheduler
(src/scheduler/distributed_pipeline_scheduler.cuh:25-139, .cu:60-511) on
torch.distributed, one process per GPU.

What it keeps from the reference: the API (DistributedConfig,
DistributedStats, upload / run_until / download, partition, rank, size,
min_local_time_step, min_global_time_step), the zone partition (slabs along
x, n = max(3, floor(L_x / rc)), zones dealt to ranks in contiguous blocks,
zone_partition.cpp:15-40,153-200), the ring (each rank talks to rank - 1 and
rank + 1 only, mpi_ring_comm.cpp:60-66), every rank holding the whole system
on its GPU (ADR 0006's full replication) while advancing only the atoms of
its own zones, and the NVT form (global KE reduced over ranks, the chain's
half step on every rank, local velocities scaled; .cu:406-452).

What is B200-first:

* The exchange carries the boundary zones' positions device to device over
  NCCL (send/recv of contiguous slices of the zone-ordered position array:
  no packing, no host staging); gloo process groups stage through host
  tensors.
* Every step is the synchronous velocity-Verlet step: local kick + drift,
  ring exchange of the boundary zones, forces of the local atoms from local
  and ghost positions (compute_morse_gpu_zone), closing local kick.  The
  reference instead steps zones whose neighbors are one step behind
  (.cu:190-216), which moves a boundary atom against a ghost that has not
  drifted yet; here a zone's force step requires its ghosts at the same
  step (the dependency check, I-2 of pipeline_scheduler.cu:93-121, counted
  in stats), so the trajectory is the single-rank one.
* Zones are re-assigned from the positions at every neighbor-list rebuild
  where an atom has left its zone's slab (the reference assigns once, at
  upload, .cu:139-190): every atom a local row lists then lies in a local or
  ghost zone, so the ghost exchange feeds every listed pair.  The criterion
  and the assignment depend on the global state only, and every per-atom
  and per-zone operation is the same whatever the rank count, so a run on N
  ranks gives the bits of the run on one rank (NVT included: the kinetic
  energy is summed per zone, then over zones in zone order).

The per-zone multi-stream schedule of the single-rank PipelineScheduler is
not reproduced: on one GPU the whole system advances as one step (the
library's FastPipelineScheduler).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import api
from ._lib import Box, MorseParams, check, lib


# --------------------------------------------------------------------------
# Zones and their partition (src/scheduler/zone.hpp, src/domain/zone_partition.*)
# --------------------------------------------------------------------------
FREE, RECEIVING, RECEIVED, READY, COMPUTING, DONE, SENDING = range(7)


@dataclass
class Zone:
    """zone.hpp:42-66: a slab of the box, its atoms [atom_offset,
    atom_offset + natoms_in_zone) of the zone-ordered arrays."""
    id: int
    lo: float
    hi: float
    atom_offset: int = 0
    natoms_in_zone: int = 0
    time_step: int = 0
    state: int = FREE
    owner_rank: int = 0


class ZonePartition:
    """zone_partition.cpp: slabs along x, their neighbors within r_list
    (periodic in x), their owner ranks."""

    def __init__(self):
        self.zones: list[Zone] = []
        self._nbrs: list[list[int]] = []
        self.lo_x = 0.0
        self.width = 1.0

    # zone_partition.cpp:15-40
    def build(self, box: Box, r_cut: float, n_zones: int = 0) -> None:
        lx = float(box.hi[0] - box.lo[0])
        self.lo_x = float(box.lo[0])
        if n_zones <= 0:
            n_zones = max(3, int(math.floor(lx / r_cut)))
        if n_zones < 3:
            raise ValueError("need at least 3 zones (periodic x)")
        self.width = lx / n_zones
        self.zones = [Zone(i, self.lo_x + i * (lx / n_zones), self.lo_x + (i + 1) * (lx / n_zones))
                      for i in range(n_zones)]
        self._nbrs = [[] for _ in range(n_zones)]

    @property
    def n_zones(self) -> int:
        return len(self.zones)

    # zone_partition.cpp:42-47 (truncation toward zero, clamped)
    def zone_of(self, x) -> np.ndarray:
        z = np.trunc((np.asarray(x, np.float64) - self.lo_x) / self.width).astype(np.int64)
        return np.clip(z, 0, self.n_zones - 1)

    def span(self, r_list: float) -> int:
        """Zone widths r_list reaches (zone_partition.cpp:128)."""
        return int(math.ceil(r_list / self.width))

    # zone_partition.cpp:124-150
    def build_zone_neighbors(self, r_list: float) -> None:
        s, n = self.span(r_list), self.n_zones
        self._nbrs = [sorted({(z + d) % n for d in range(-s, s + 1)}) for z in range(n)]

    def zone_neighbors(self, z: int) -> list:
        return self._nbrs[z]

    # zone_partition.cpp:153-169: as even as possible, the first
    # n_zones % n_ranks ranks one zone more, contiguous blocks in rank order
    def assign_to_ranks(self, n_ranks: int) -> None:
        if n_ranks < 1:
            raise ValueError("need at least 1 rank")
        if self.n_zones < n_ranks:
            raise ValueError("need at least as many zones as ranks")
        base, rem = divmod(self.n_zones, n_ranks)
        z = 0
        for r in range(n_ranks):
            for _ in range(base + (1 if r < rem else 0)):
                self.zones[z].owner_rank = r
                z += 1

    def owner_rank(self, z: int) -> int:
        return self.zones[z].owner_rank

    def is_local(self, z: int, rank: int) -> bool:
        return self.zones[z].owner_rank == rank

    def first_zone_of_rank(self, r: int) -> int:
        for z in self.zones:
            if z.owner_rank == r:
                return z.id
        return self.n_zones

    def n_zones_of_rank(self, r: int) -> int:
        return sum(1 for z in self.zones if z.owner_rank == r)

    # zone_partition.cpp:187-200
    def ghost_zones(self, rank: int) -> list:
        g = {nz for z in range(self.n_zones) if self.is_local(z, rank)
             for nz in self._nbrs[z] if not self.is_local(nz, rank)}
        return sorted(g)

    def assign_atoms(self, x) -> np.ndarray:
        """zone_partition.cpp:49-121: the permutation that groups atoms by
        zone (counting sort, input order within a zone); records each zone's
        offset and count.  Returns perm: new index k holds old atom perm[k]."""
        z = self.zone_of(x)
        perm = np.argsort(z, kind="stable").astype(np.int64)
        counts = np.bincount(z, minlength=self.n_zones)
        offs = np.concatenate([[0], np.cumsum(counts)[:-1]])
        for zone, o, c in zip(self.zones, offs, counts):
            zone.atom_offset, zone.natoms_in_zone = int(o), int(c)
        return perm

    def atom_range(self, z0: int, z1: int) -> tuple:
        """Atoms of zones [z0, z1) (z1 > z0, no wrap)."""
        a = self.zones[z0].atom_offset
        b = self.zones[z1 - 1].atom_offset + self.zones[z1 - 1].natoms_in_zone
        return a, b


# --------------------------------------------------------------------------
# The ring exchange
# --------------------------------------------------------------------------
def _runs(zones) -> list:
    """Ordered zone ids as runs (za, zb) of consecutive ids."""
    out = []
    for z in zones:
        if out and out[-1][1] == z:
            out[-1] = (out[-1][0], z + 1)
        else:
            out.append((z, z + 1))
    return out


def _side_ghosts(part: ZonePartition, rank: int, span: int) -> tuple:
    """The ghost zones below a rank's block (z0 - span .. z0 - 1) and above it
    (z1 .. z1 + span - 1), periodic in x, local zones and repeats left out,
    in that order."""
    nz = part.n_zones
    z0 = part.first_zone_of_rank(rank)
    z1 = z0 + part.n_zones_of_rank(rank)
    lo, hi = [], []
    for k in range(span, 0, -1):
        z = (z0 - k) % nz
        if not part.is_local(z, rank) and z not in lo:
            lo.append(z)
    for k in range(span):
        z = (z1 + k) % nz
        if not part.is_local(z, rank) and z not in hi:
            hi.append(z)
    return lo, hi


@dataclass
class RingPlan:
    """A rank's part of the ring exchange, as runs of zones: its lower ghosts
    come from the previous rank and its upper ghosts from the next; it sends
    the next rank that rank's lower ghosts and the previous rank that rank's
    upper ghosts."""
    rank: int
    world: int
    prev: int
    next: int
    local: tuple = (0, 0)
    to_next: list = field(default_factory=list)
    to_prev: list = field(default_factory=list)
    from_prev: list = field(default_factory=list)
    from_next: list = field(default_factory=list)


def ring_plan(part: ZonePartition, rank: int, world: int, span: int) -> RingPlan:
    """The exchange of every rank is fixed by the partition alone, so sender
    and receiver derive the same runs.  Every ghost zone must belong to a ring
    neighbor (lower ghosts to the previous rank, upper to the next)."""
    z0 = part.first_zone_of_rank(rank)
    prev, nxt = (rank - 1) % world, (rank + 1) % world
    p = RingPlan(rank, world, prev, nxt, local=(z0, z0 + part.n_zones_of_rank(rank)))
    if world == 1:
        return p
    for r in range(world):
        lo, hi = _side_ghosts(part, r, span)
        bad = ([z for z in lo if part.owner_rank(z) != (r - 1) % world] +
               [z for z in hi if part.owner_rank(z) != (r + 1) % world])
        if bad:
            raise ValueError(
                f"rank {r} needs zones {bad} from ranks other than its ring neighbors: each rank "
                f"should own at least {span} zones (r_cut + r_skin spans {span} zone widths); "
                "use fewer ranks or more zones")
    lo, hi = _side_ghosts(part, rank, span)
    p.from_prev, p.from_next = _runs(lo), _runs(hi)
    p.to_next = _runs(_side_ghosts(part, nxt, span)[0])
    p.to_prev = _runs(_side_ghosts(part, prev, span)[1])
    return p


def ring_exchange(dist, group, arr, part: ZonePartition, plan: RingPlan, ts_local: int):
    """Sends the rows of arr (zone-ordered, [n, k]) that the ring neighbors
    hold as ghosts and receives this rank's ghost rows into arr, in place;
    returns the time steps the two neighbors reported (the dependency
    check's ghost time steps).  Device tensors go directly under NCCL;
    otherwise rows are staged through host tensors.

    One message per direction: a time step, then one tensor per zone run.
    Operation order, the same on every rank: to next, to prev, from prev,
    from next.  With two ranks (prev == next) point-to-point messages
    between one pair match in order, and the peer's first receive (its
    lower ghosts) is this rank's first send (the peer's lower ghosts)."""
    import torch
    if plan.world == 1:
        return ts_local, ts_local
    direct = arr.is_cuda and dist.get_backend(group) == "nccl"
    dev = arr.device if direct else torch.device("cpu")

    def rows(za, zb):
        a, b = part.atom_range(za, zb)
        return arr[a:b]

    ops, fills, ts_in = [], [], []
    for runs, peer, tag in ((plan.to_next, plan.next, 1), (plan.to_prev, plan.prev, 2)):
        ops.append(dist.P2POp(dist.isend, torch.full((1,), ts_local, dtype=torch.int64,
                                                     device=dev), peer, group, tag))
        for k, (za, zb) in enumerate(runs):
            t = rows(za, zb)
            ops.append(dist.P2POp(dist.isend, t if direct else t.cpu(), peer, group,
                                  100 * tag + k))
    for runs, peer, tag in ((plan.from_prev, plan.prev, 1), (plan.from_next, plan.next, 2)):
        t = torch.empty(1, dtype=torch.int64, device=dev)
        ts_in.append(t)
        ops.append(dist.P2POp(dist.irecv, t, peer, group, tag))
        for k, (za, zb) in enumerate(runs):
            dst = rows(za, zb)
            buf = dst if direct else torch.empty(dst.shape, dtype=dst.dtype)
            if not direct:
                fills.append((dst, buf))
            ops.append(dist.P2POp(dist.irecv, buf, peer, group, 100 * tag + k))
    for w in dist.batch_isend_irecv(ops):
        w.wait()
    for dst, buf in fills:
        dst.copy_(buf)
    return int(ts_in[0].item()), int(ts_in[1].item())


# --------------------------------------------------------------------------
# The scheduler
# --------------------------------------------------------------------------
@dataclass
class DistributedConfig:
    """distributed_pipeline_scheduler.cuh:27-39, plus the force precision
    (the reference picks it at build time)."""
    dt: float = 0.001
    r_skin: float = 1.0
    n_zones: int = 0
    n_streams: int = 4          # accepted; one stream per rank here
    rebuild_every: int = 10
    deterministic: bool = False  # accepted; every run here is deterministic
    t_target: float = 0.0
    t_period: float = 0.1
    nhc_length: int = 3
    precision: str = "fp64"


@dataclass
class DistributedStats:
    """distributed_pipeline_scheduler.cuh:41-47.  kernel_launches counts zone
    steps (one per local zone per step, as the reference counts
    launch_zone_step); exchanges counts ring exchanges; rezones (no
    reference counterpart) counts zone re-assignments at rebuilds."""
    kernel_launches: int = 0
    dep_check_calls: int = 0
    dep_check_failures: int = 0
    ticks: int = 0
    exchanges: int = 0
    rezones: int = 0


@dataclass
class _State:
    pos: object = None
    vel: object = None
    forces: object = None
    types: object = None
    ids: object = None
    masses: object = None


class DistributedPipelineScheduler:
    """DistributedPipelineScheduler(box, natoms, MorseParams, DistributedConfig,
    group): every rank of the process group (dist.group.WORLD when None)
    constructs it with the same arguments, uploads the same system and makes
    the same calls in the same order (upload, run_until, download and
    energies are collective).  Each rank uses its current CUDA device."""

    def __init__(self, box: Box, natoms: int, params: MorseParams,
                 cfg: DistributedConfig | None = None, group=None, dist=None):
        import torch
        if dist is None:
            import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.cfg = cfg or DistributedConfig()
        self.box = box
        self.params = params
        self.natoms = int(natoms)
        self._rank = dist.get_rank(group) if dist.is_initialized() else 0
        self._size = dist.get_world_size(group) if dist.is_initialized() else 1
        if self._size > 1 and not dist.is_initialized():
            raise RuntimeError("a process group is needed for more than one rank")
        r_list = params.rc + self.cfg.r_skin
        self.part = ZonePartition()
        self.part.build(box, params.rc, self.cfg.n_zones)
        self.part.assign_to_ranks(self._size)
        self.part.build_zone_neighbors(r_list)
        self.span = self.part.span(r_list)
        self.plan = ring_plan(self.part, self._rank, self._size, self.span)
        self._ghosts = self.part.ghost_zones(self._rank)
        self._zone_calls = None
        self.stats_ = DistributedStats()
        self.dev = torch.device("cuda", torch.cuda.current_device())
        self.s = _State()
        self.nlist = api.DeviceNeighborList()
        self.nhc = None
        if self.cfg.t_target > 0:
            self.nhc = api.NoseHooverChain(self.cfg.t_target, self.cfg.t_period,
                                           self.cfg.nhc_length, self.cfg.dt, 3 * self.natoms - 3)
        self._step = 0
        self._since = 0
        self._initialized = False
        self._uploaded = False

    # --- reference accessors ----------------------------------------------
    def partition(self) -> ZonePartition:
        return self.part

    def stats(self) -> DistributedStats:
        return self.stats_

    def rank(self) -> int:
        return self._rank

    def size(self) -> int:
        return self._size

    def min_local_time_step(self) -> int:
        z0, z1 = self.plan.local
        return min(self.part.zones[z].time_step for z in range(z0, z1))

    def min_global_time_step(self) -> int:
        """All ranks' minimum (an all_reduce(min), .cu:470-475)."""
        v = self.min_local_time_step()
        if self._size == 1:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.int64, device=self._coll_device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN, group=self.group)
        return int(t.item())

    # --- helpers ------------------------------------------------------------
    def _coll_device(self):
        import torch
        if self._size > 1 and self.dist.get_backend(self.group) == "nccl":
            return self.dev
        return torch.device("cpu")

    def _fdtype(self):
        import torch
        return torch.float64 if self.cfg.precision == "fp64" else torch.float32

    def _local(self) -> tuple:
        return self.part.atom_range(*self.plan.local)

    def _set_state(self, pos, vel, forces, types, ids):
        """Host arrays in zone order -> device."""
        import torch
        d = self.dev
        self.s.pos = torch.from_numpy(np.ascontiguousarray(pos, np.float64)).to(d)
        self.s.vel = torch.from_numpy(np.ascontiguousarray(vel, np.float64)).to(d)
        self.s.forces = torch.from_numpy(np.ascontiguousarray(forces)).to(d, self._fdtype())
        self.s.types = torch.from_numpy(np.ascontiguousarray(types, np.int32)).to(d)
        self.s.ids = torch.from_numpy(np.ascontiguousarray(ids, np.int32)).to(d)

    def _zone(self, perm, pos, vel, forces, types, ids):
        return pos[perm], vel[perm], forces[perm], types[perm], ids[perm]

    # --- upload / download ---------------------------------------------------
    def upload(self, positions, velocities, forces, types, ids, masses, n_masses=None):
        """.cu:139-190: the system grouped by zone on every rank."""
        import torch
        n = self.natoms
        pos = np.asarray(positions, np.float64).reshape(n, 3)
        vel = np.asarray(velocities, np.float64).reshape(n, 3)
        frc = (np.zeros((n, 3)) if forces is None else np.asarray(forces).reshape(n, 3))
        typ = np.asarray(types, np.int32).reshape(n)
        ids_ = (np.arange(1, n + 1, dtype=np.int32) if ids is None
                else np.asarray(ids, np.int32).reshape(n))
        m = np.asarray(masses, np.float64).reshape(-1)
        if n_masses is not None:
            m = m[:int(n_masses)]
        if typ.size and (typ.min() < 1 or typ.max() >= m.size):
            raise ValueError("atom type out of range of masses")
        perm = self.part.assign_atoms(pos[:, 0])
        self._set_state(*self._zone(perm, pos, vel, frc.astype(np.float64), typ, ids_))
        self.s.masses = torch.from_numpy(m.copy()).to(self.dev)
        for z in self.part.zones:
            z.state, z.time_step = READY, 0
        self._step = 0
        self._since = 0
        self._initialized = False
        self._uploaded = True

    def _gather_full(self):
        """Every rank's local atoms to every rank (one all_gather per array of
        rank-sized blocks padded to the largest), so the device arrays hold
        the current state of the whole system."""
        if self._size == 1:
            return
        import torch
        blocks = [self.part.atom_range(self.part.first_zone_of_rank(r),
                                       self.part.first_zone_of_rank(r) +
                                       self.part.n_zones_of_rank(r))
                  for r in range(self._size)]
        mx = max(b - a for a, b in blocks)
        direct = self.dist.get_backend(self.group) == "nccl"
        a0, b0 = blocks[self._rank]
        for name in ("pos", "vel", "forces", "types", "ids"):
            arr = getattr(self.s, name)
            shape = (mx,) + tuple(arr.shape[1:])
            mine = torch.zeros(shape, dtype=arr.dtype, device=arr.device if direct else "cpu")
            mine[:b0 - a0].copy_(arr[a0:b0])
            outs = [torch.empty_like(mine) for _ in range(self._size)]
            self.dist.all_gather(outs, mine, group=self.group)
            for r, (a, b) in enumerate(blocks):
                if r != self._rank:
                    arr[a:b].copy_(outs[r][:b - a])

    def download(self):
        """The whole system in its current zone order (collective): positions,
        velocities, forces, types, ids as host arrays (.cu:493-505)."""
        self._require_uploaded()
        self._gather_full()
        s = self.s
        return (s.pos.cpu().numpy(), s.vel.cpu().numpy(), s.forces.cpu().numpy(),
                s.types.cpu().numpy(), s.ids.cpu().numpy())

    def _require_uploaded(self):
        if not self._uploaded:
            raise RuntimeError("upload before run_until / download")

    # --- zone steps ------------------------------------------------------------
    def _rebuild(self):
        """The neighbor list over the whole (current) system, after
        re-assigning zones when an atom has left its slab."""
        self._gather_full()
        x = self.s.pos[:, 0].cpu().numpy()
        assigned = np.repeat(np.arange(self.part.n_zones),
                             [z.natoms_in_zone for z in self.part.zones])
        if np.any(self.part.zone_of(x) != assigned):
            perm = self.part.assign_atoms(x)
            p = __import__("torch").from_numpy(perm).to(self.dev)
            for name in ("pos", "vel", "forces", "types", "ids"):
                setattr(self.s, name, getattr(self.s, name).index_select(0, p).contiguous())
            self.stats_.rezones += 1
        self.nlist.build(self.s.pos, self.natoms, self.box, self.params.rc, self.cfg.r_skin)
        self._zone_calls = self._prepare_zone_calls()

    def _prepare_zone_calls(self):
        """The argument lists of the local zones' force calls, fixed until
        the next rebuild (list and state arrays are not reallocated between
        rebuilds)."""
        nb, off, cnt = self.nlist._get()[:3]
        fn = lib().tdmd_morse_compute_zone
        head = (C.c_void_p(self.s.pos.data_ptr()), C.c_void_p(self.s.forces.data_ptr()),
                api._prec(self.cfg.precision), C.c_void_p(nb), C.c_void_p(off), C.c_void_p(cnt))
        tail = (C.byref(self.box), C.byref(self.params), None, None, None)
        calls = []
        for z in range(*self.plan.local):
            zn = self.part.zones[z]
            if zn.natoms_in_zone:
                calls.append(head + (zn.atom_offset, zn.natoms_in_zone) + tail)
        return fn, calls

    def _local_forces(self):
        """One zone call per local zone (launch_zone_step's force call,
        pipeline_scheduler.cu:142-146): each zone's launch shape follows its
        own atom count, the same for every rank count."""
        a, b = self._local()
        api.device_zero_forces(self.s.forces[a:b], b - a)
        fn, calls = self._zone_calls
        for args in calls:
            rc = fn(*args)
            if rc != 0:
                check(rc)

    def _check_deps(self, ghost_ts):
        """I-2 (pipeline_scheduler.cu:93-121): each local zone's ghosts are
        at its own step before its forces are computed."""
        z0, z1 = self.plan.local
        for z in range(z0, z1):
            self.stats_.dep_check_calls += 1
            if min(ghost_ts) < self.part.zones[z].time_step + 1:
                self.stats_.dep_check_failures += 1
                raise RuntimeError(f"zone {z}: ghost zones behind (time steps {ghost_ts})")

    def _zone_ke(self) -> float:
        """Kinetic energy summed per zone, then over the zones in zone order
        (the same sum on every rank and for every rank count)."""
        import torch
        nz = self.part.n_zones
        ke = torch.zeros(nz, dtype=torch.float64)
        z0, z1 = self.plan.local
        for z in range(z0, z1):
            zn = self.part.zones[z]
            a, b = zn.atom_offset, zn.atom_offset + zn.natoms_in_zone
            if b > a:
                ke[z] = api.device_compute_ke(self.s.vel[a:b], self.s.types[a:b], self.s.masses,
                                              b - a)
        if self._size > 1:
            t = ke.to(self._coll_device())
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
            ke = t.cpu()
        tot = 0.0
        for v in ke.tolist():
            tot += v
        return tot

    def _thermostat(self):
        scale = self.nhc.half_step(self._zone_ke())
        a, b = self._local()
        api.device_scale_velocities(self.s.vel[a:b], b - a, scale)

    def _initial_forces(self):
        self._rebuild()
        self._local_forces()
        self._since = 0
        self._initialized = True

    def run_until(self, target_step: int):
        """Advances every zone to target_step (collective; run_until(0)
        computes the forces only)."""
        self._require_uploaded()
        if not self._initialized:
            self._initial_forces()
        dt = self.cfg.dt
        while self._step < target_step:
            if self.nhc is not None:
                self._thermostat()
            a, b = self._local()
            s = self.s
            api.device_fused_half_kick_drift(s.vel[a:b], s.pos[a:b], s.forces[a:b],
                                             s.types[a:b], s.masses, b - a, dt, self.box)
            ghost_ts = ring_exchange(self.dist, self.group, s.pos, self.part, self.plan,
                                     self._step + 1)
            if self._size > 1:
                self.stats_.exchanges += 1
            self._check_deps(ghost_ts)
            # the library scheduler's schedule: after the kick-drift of the
            # step that follows rebuild_every steps on one list
            if self._since >= self.cfg.rebuild_every:
                self._rebuild()
                self._since = 0
            self._since += 1
            self._local_forces()
            a, b = self._local()
            api.device_half_kick(s.vel[a:b], s.forces[a:b], s.types[a:b], s.masses, b - a, dt)
            if self.nhc is not None:
                self._thermostat()
            self._step += 1
            z0, z1 = self.plan.local
            for z in range(z0, z1):
                self.part.zones[z].time_step = self._step
            for z in self._ghosts:
                self.part.zones[z].time_step = self._step
            self.stats_.kernel_launches += z1 - z0
            self.stats_.ticks += 1
        import torch
        torch.cuda.synchronize(self.dev)

    def current_step(self) -> int:
        return self._step

    def energies(self):
        """(potential, kinetic) energy of the whole system (collective):
        per-zone sums added in zone order."""
        import torch
        self._require_uploaded()
        if not self._initialized:
            self._initial_forces()
        nz = self.part.n_zones
        pe = torch.zeros(nz, dtype=torch.float64)
        z0, z1 = self.plan.local
        scratch = torch.zeros_like(self.s.forces)
        for z in range(z0, z1):
            zn = self.part.zones[z]
            if zn.natoms_in_zone:
                e = torch.zeros(1, dtype=torch.float64, device=self.dev)
                api.compute_morse_gpu_zone(self.s.pos, scratch, self.nlist.d_neighbors(),
                                           self.nlist.d_offsets(), self.nlist.d_counts(),
                                           zn.atom_offset, zn.natoms_in_zone, self.box,
                                           self.params, d_energy=e,
                                           precision=self.cfg.precision)
                pe[z] = e.item()
        if self._size > 1:
            t = pe.to(self._coll_device())
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
            pe = t.cpu()
        tot = 0.0
        for v in pe.tolist():
            tot += v
        return tot, self._zone_ke()
