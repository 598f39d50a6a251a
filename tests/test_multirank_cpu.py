"""Multi-GPU host logic on CPU: replica sharding (longest-processing-time
balance by atom count) with the per-replica results gathered back in order,
force matching sharded by snapshot (one all_reduce of the weighted loss and
gradient per evaluation), and the max/sum-over-ranks reductions, run as two
gloo ranks on 127.0.0.1; the bench's reference arm under torchrun (rank 0
reports, other ranks exit without work).  The per-rank work is the oracle's
on the CPU; only the host logic around it is under test (unmeasured on
more than one GPU)."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import numpy as np
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_lpt_partition_balances_replicas():
    from tdmd_claude_b200 import workloads as W
    from tdmd_claude_b200.replicas import lpt_partition
    sizes = [s.n for s in W.replica_set(64, seed=5)]
    for parts in (1, 2, 3, 8):
        bins = lpt_partition(sizes, parts)
        flat = sorted(i for b in bins for i in b)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in b) for b in bins]
        # LPT: the heaviest bin exceeds the mean by at most the largest item
        assert max(loads) - np.mean(loads) <= max(sizes)
    assert lpt_partition([5, 3, 2], 2) == [[0], [1, 2]]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from tdmd_claude_b200.replicas import max_over_ranks, sum_over_ranks
    mx = max_over_ranks(1.5 + rank, dist)
    sm = sum_over_ranks(10 * (rank + 1), dist)
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump({"max": mx, "sum": sm}, f)


def test_reductions_over_two_gloo_ranks(tmp_path):
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        got = json.load(open(tmp_path / f"r{r}.json"))
        assert got == {"max": 2.5, "sum": 30.0}


def _fm_problem():
    """6 snapshots of a jittered 3^3 Cu FCC (108 atoms), Morse rc 5.0 and the
    analytic Cu EAM; targets from perturbed parameters (FP64 oracle)."""
    from oracle import oracle as O
    from tdmd_claude_b200 import workloads as W
    rng = np.random.default_rng(3)
    base = W.fcc_lattice(3, 3, 3, 3.615)
    L = 3 * 3.615
    pos = np.stack([np.mod(base + rng.uniform(-0.15, 0.15, base.shape), L) for _ in range(6)])
    lo, hi = (0.0, 0.0, 0.0), (L, L, L)
    morse = (0.3429, 1.3588, 2.866, 5.0)
    tm = np.stack([O.morse_forces(p, lo, hi, 0.33, 1.40, 2.85, 5.0, 0.0)[1] for p in pos])
    t = W.cu_eam_tables()
    oe = O.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    te = np.stack([oe.forces(p, np.ones(len(p), np.int32), lo, hi, 0.0)["forces"] * 1.03
                   for p in pos])
    return pos, lo, hi, morse, tm, te, oe


class _OracleShard:
    """The oracle's FP64 loss and gradient on one shard, with ForceMatch's
    morse / eam interface on CPU tensors."""

    def __init__(self, pos, lo, hi, morse, tm, te, oe):
        self.pos, self.lo, self.hi, self.morse_p = pos, lo, hi, morse
        self.tm, self.te, self.oe = tm, te, oe

    def morse(self, params, loss, grad=None, forces=None):
        from oracle import oracle as O
        D, a, r0 = params.tolist()
        val, g = O.morse_fm_loss_grad(self.pos, self.lo, self.hi, D, a, r0, self.morse_p[3],
                                      self.tm)
        loss.fill_(val)
        if grad is not None:
            grad.copy_(torch.from_numpy(g))

    def eam(self, tables, F, rho, phi, loss, gF=None, grho=None, gphi=None, forces=None):
        val, a, b, c = self.oe.fm_loss_grad(self.pos, np.ones(self.pos.shape[1], np.int32),
                                            self.lo, self.hi, self.te)
        loss.fill_(val)
        for t, v in ((gF, a), (grho, b), (gphi, c)):
            if t is not None:
                t.copy_(torch.from_numpy(v.reshape(t.shape)))


def _fm_rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from tdmd_claude_b200.fitting import ShardedForceMatch, morse_loss, snapshot_shard
    pos, lo, hi, morse, tm, te, oe = _fm_problem()
    sh = snapshot_shard(len(pos), rank, world)
    local = _OracleShard(pos[sh.start:sh.stop], lo, hi, morse, tm[sh.start:sh.stop],
                         te[sh.start:sh.stop], oe)
    fm = ShardedForceMatch(local, len(sh), len(pos), dist)
    prm = torch.tensor(morse[:3], dtype=torch.float64, requires_grad=True)
    loss = morse_loss(prm, fm)
    loss.backward()
    ml, mg = float(loss.item()), prm.grad.tolist()
    nt = 1
    gF = torch.zeros((nt, 4 * (oe.nrho - 1)), dtype=torch.float64)
    gr = torch.zeros((nt, 4 * (oe.nr - 1)), dtype=torch.float64)
    gp = torch.zeros((1, 4 * (oe.nr - 1)), dtype=torch.float64)
    el = torch.zeros(1, dtype=torch.float64)
    fm.eam({}, None, None, None, el, gF, gr, gp)
    dist.barrier()
    dist.destroy_process_group()
    np.savez(os.path.join(out_dir, f"fm{rank}.npz"), ml=ml, mg=np.array(mg), el=el.numpy(),
             gF=gF.numpy(), gr=gr.numpy(), gp=gp.numpy(), shard=np.array([sh.start, sh.stop]))


def test_sharded_force_matching_two_gloo_ranks(tmp_path):
    """Each rank evaluates the oracle's loss and gradient on its snapshots;
    after the one all_reduce they equal the single-rank oracle on all
    snapshots to 1e-12 (Morse through the autograd wrapper, EAM raw)."""
    from oracle import oracle as O
    port = _free_port()
    mp.start_processes(_fm_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    pos, lo, hi, morse, tm, te, oe = _fm_problem()
    L, g = O.morse_fm_loss_grad(pos, lo, hi, *morse, tm)
    eL, eF, er, ep = oe.fm_loss_grad(pos, np.ones(pos.shape[1], np.int32), lo, hi, te)
    shards = []
    for r in range(2):
        d = np.load(tmp_path / f"fm{r}.npz")
        shards.append(tuple(d["shard"]))
        assert abs(float(d["ml"]) - L) <= 1e-12 * abs(L)
        assert np.abs(d["mg"] - g).max() <= 1e-12 * np.abs(g).max()
        assert abs(float(d["el"][0]) - eL) <= 1e-12 * abs(eL)
        for got, want in ((d["gF"], eF), (d["gr"], er), (d["gp"], ep)):
            assert np.abs(got.reshape(want.shape) - want).max() <= 1e-12 * np.abs(want).max()
    assert shards == [(0, 3), (3, 6)]


def test_snapshot_shard_covers_every_snapshot():
    from tdmd_claude_b200.fitting import snapshot_shard
    for n, w in ((64, 1), (64, 3), (7, 4), (5, 5)):
        got = [i for r in range(w) for i in snapshot_shard(n, r, w)]
        assert got == list(range(n))
        sizes = [len(snapshot_shard(n, r, w)) for r in range(w)]
        assert max(sizes) - min(sizes) <= 1


def _replica_rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from oracle import oracle as O
    from tdmd_claude_b200 import workloads as W
    from tdmd_claude_b200.replicas import gather_by_replica, lpt_partition
    systems = W.replica_set(12, seed=9, nmin=4, nmax=5)
    mine = lpt_partition([s.n for s in systems], world)[rank]
    D, a, r0, rc = W.MORSE_CU
    vals = [O.morse_forces(systems[i].positions, systems[i].lo, systems[i].hi, D, a, r0, rc,
                           0.3)[0] for i in mine]
    got = gather_by_replica(vals, mine, len(systems), dist)
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rep{rank}.json"), "w") as f:
        json.dump({"mine": list(mine), "pe": got}, f)


def test_lpt_shards_gather_back_in_replica_order(tmp_path):
    """Replicas split by LPT over two ranks; each rank's per-replica Morse
    energies (oracle), gathered, equal the unsharded list in order."""
    from oracle import oracle as O
    from tdmd_claude_b200 import workloads as W
    port = _free_port()
    mp.start_processes(_replica_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    systems = W.replica_set(12, seed=9, nmin=4, nmax=5)
    D, a, r0, rc = W.MORSE_CU
    want = [O.morse_forces(s.positions, s.lo, s.hi, D, a, r0, rc, 0.3)[0] for s in systems]
    outs = [json.load(open(tmp_path / f"rep{r}.json")) for r in range(2)]
    assert sorted(outs[0]["mine"] + outs[1]["mine"]) == list(range(12))
    assert outs[0]["mine"] and outs[1]["mine"]
    for o in outs:
        assert o["pe"] == want


def test_reference_arm_under_torchrun_env(tmp_path):
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--gpus", "2", "--steps", "1", "--warmup", "3"],
                         capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0 and out.stdout.strip() == ""


def test_reference_arm_prints_its_line():
    """bench.py --impl reference on rank 0: one JSON line with the arm's
    contract keys (the reference CPU loop, a bounded sample)."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "3", "--cpu-cores", "2"],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "atom-steps/s" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] == 2
    assert d["config"]["processes"] == 2 and len(d["config"]["per_process_loop_s"]) == 2
