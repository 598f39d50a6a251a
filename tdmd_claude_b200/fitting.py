"""Force-matching fits of Morse parameters and EAM spline coefficients.

The loss and its gradient come from the C ABI (tdmd_fit_*: the adjoint of
the force expressions on the GPU, FP64 accumulation).  torch supplies device
tensors, the optimizer and the autograd plumbing only: MorseLoss and EamLoss
are torch.autograd.Functions whose forward runs the loss + gradient kernels
once and whose backward scales that gradient.

No reference counterpart (the reference computes no gradients); the force
definitions are those of src/potentials/morse.hpp:37-55 and
src/potentials/eam_alloy.cpp:196-295.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from ._lib import TDMD_FP64, TDMD_MIXED, Box, call, lib


def _dptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _cur_stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class ForceMatch:
    """Snapshots positions[s, n, 3] (one box, 1-based types[s, n] or [n]),
    neighbor lists with r_list = cutoff built once on the device."""

    def __init__(self, positions, types, box: Box, cutoff: float, precision: str = "fp64"):
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        self.nsnap, self.natoms = pos.shape[0], pos.shape[1]
        typ = np.ascontiguousarray(np.broadcast_to(
            np.asarray(types, np.int32).reshape(-1, self.natoms), (self.nsnap, self.natoms)),
            dtype=np.int32)
        self.cutoff = float(cutoff)
        self.precision = precision
        h = C.c_void_p()
        call("tdmd_fit_create", self.nsnap, self.natoms, C.byref(box),
             pos.ctypes.data_as(C.c_void_p), typ.ctypes.data_as(C.c_void_p), self.cutoff,
             TDMD_FP64 if precision == "fp64" else TDMD_MIXED, C.byref(h))
        self._h = h

    def __del__(self):
        self.close()

    def close(self):
        if getattr(self, "_h", None):
            try:
                lib().tdmd_fit_destroy(self._h)
            except Exception:
                pass
            self._h = None

    def set_targets(self, targets):
        t = np.ascontiguousarray(targets, dtype=np.float64)
        assert t.size == 3 * self.nsnap * self.natoms
        call("tdmd_fit_set_targets", self._h, t.ctypes.data_as(C.c_void_p))

    # raw calls on device tensors (float64, cuda) ---------------------------
    def morse(self, params, loss, grad=None, forces=None):
        call("tdmd_fit_morse", self._h, _dptr(params), _dptr(loss), _dptr(grad), _dptr(forces),
             _cur_stream())

    def eam(self, tables: dict, F, rho, phi, loss, gF=None, grho=None, gphi=None, forces=None):
        call("tdmd_fit_eam", self._h, int(tables["ntypes"]), int(tables["nrho"]),
             float(tables["drho"]), int(tables["nr"]), float(tables["dr"]), _dptr(F),
             _dptr(rho), _dptr(phi), _dptr(loss), _dptr(gF), _dptr(grho), _dptr(gphi),
             _dptr(forces), _cur_stream())

    def morse_forces(self, params):
        import torch
        p = torch.as_tensor(np.asarray(params, np.float64), device="cuda")
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        f = torch.zeros(self.nsnap * self.natoms * 3, dtype=torch.float64, device="cuda")
        if not getattr(self, "_has_targets", False):
            self.set_targets(np.zeros(3 * self.nsnap * self.natoms))
            self._has_targets = True
        self.morse(p, loss, None, f)
        return f.cpu().numpy().reshape(self.nsnap, self.natoms, 3)

    def eam_forces(self, tables: dict, F, rho, phi):
        import torch
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        f = torch.zeros(self.nsnap * self.natoms * 3, dtype=torch.float64, device="cuda")
        if not getattr(self, "_has_targets", False):
            self.set_targets(np.zeros(3 * self.nsnap * self.natoms))
            self._has_targets = True
        self.eam(tables, F, rho, phi, loss, forces=f)
        return f.cpu().numpy().reshape(self.nsnap, self.natoms, 3)


def snapshot_shard(nsnap: int, rank: int, world: int) -> range:
    """The contiguous, balanced slice of snapshot indices that `rank` of
    `world` owns (the first nsnap % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    base, extra = divmod(int(nsnap), world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


class ShardedForceMatch:
    """Force matching sharded by snapshot over a process group.

    Each rank evaluates the loss and gradient of its own snapshots (a
    ForceMatch, or any object with the same morse / eam methods, on the
    rank's shard).  The loss is a mean over all atoms of all snapshots, so
    the global loss and gradient are the shard values weighted by
    w_r = nsnap_r / nsnap, summed over ranks: one all_reduce(sum) of the
    packed vector w_r [L_r, gradient_r] per evaluation (NCCL on GPUs, gloo
    on CPU tensors).  Predicted forces stay per shard.  The morse / eam
    methods take the same arguments as ForceMatch's, so MorseLoss / EamLoss
    (and adam_fit) run unchanged on top of it; every rank must make the same
    calls in the same order.

    No reference counterpart (the reference computes no gradients); its
    only multi-rank reduction is the scalar MPI_Allreduce of the distributed
    scheduler (src/scheduler/distributed_pipeline_scheduler.cu:432,453)."""

    def __init__(self, local, nsnap_local: int, nsnap_total: int, dist=None, group=None):
        self.local = local
        self.nsnap_local = int(nsnap_local)
        self.nsnap_total = int(nsnap_total)
        self.weight = self.nsnap_local / self.nsnap_total
        self.dist = dist
        self.group = group

    @classmethod
    def from_snapshots(cls, positions, types, box: Box, cutoff: float, precision="fp64",
                       dist=None, group=None):
        """All ranks pass the same snapshots[nsnap, n, 3] (and types); each
        builds a ForceMatch on its own shard only."""
        pos = np.asarray(positions, np.float64)
        nsnap, n = pos.shape[0], pos.shape[1]
        rank = dist.get_rank(group) if dist is not None else 0
        world = dist.get_world_size(group) if dist is not None else 1
        sh = snapshot_shard(nsnap, rank, world)
        if len(sh) == 0:
            raise ValueError("more ranks than snapshots")
        typ = np.asarray(types, np.int32).reshape(-1, n)
        typ = typ[sh.start:sh.stop] if typ.shape[0] == nsnap else typ
        fm = ForceMatch(pos[sh.start:sh.stop], typ, box, cutoff, precision)
        return cls(fm, len(sh), nsnap, dist, group)

    def set_targets(self, targets_local):
        """Targets of this rank's snapshots only ([nsnap_local, n, 3])."""
        self.local.set_targets(targets_local)

    def _reduce(self, loss, grads):
        import torch
        parts = [loss.reshape(-1)] + [g.reshape(-1) for g in grads if g is not None]
        buf = torch.cat(parts) * self.weight
        if self.dist is not None:
            self.dist.all_reduce(buf, op=self.dist.ReduceOp.SUM, group=self.group)
        off = 0
        for t in [loss] + [g for g in grads if g is not None]:
            k = t.numel()
            t.copy_(buf[off:off + k].reshape(t.shape))
            off += k

    def morse(self, params, loss, grad=None, forces=None):
        self.local.morse(params, loss, grad, forces)
        self._reduce(loss, [grad])

    def eam(self, tables: dict, F, rho, phi, loss, gF=None, grho=None, gphi=None, forces=None):
        self.local.eam(tables, F, rho, phi, loss, gF, grho, gphi, forces)
        self._reduce(loss, [gF, grho, gphi])

    def close(self):
        if hasattr(self.local, "close"):
            self.local.close()


def _autograd():
    import torch

    class MorseLoss(torch.autograd.Function):
        """loss(params[3] = D, alpha, r0) with the adjoint gradient."""

        @staticmethod
        def forward(ctx, params, fm):
            loss = torch.empty(1, dtype=torch.float64, device=params.device)
            grad = torch.empty(3, dtype=torch.float64, device=params.device)
            fm.morse(params.detach().contiguous(), loss, grad)
            ctx.save_for_backward(grad)
            return loss.reshape(())

        @staticmethod
        def backward(ctx, gout):
            (grad,) = ctx.saved_tensors
            return gout * grad, None

    class EamLoss(torch.autograd.Function):
        """loss(F, rho, phi spline coefficients) with the adjoint gradient."""

        @staticmethod
        def forward(ctx, F, rho, phi, fm, tables):
            loss = torch.empty(1, dtype=torch.float64, device=F.device)
            gF, gr, gp = torch.empty_like(F), torch.empty_like(rho), torch.empty_like(phi)
            fm.eam(tables, F.detach().contiguous(), rho.detach().contiguous(),
                   phi.detach().contiguous(), loss, gF, gr, gp)
            ctx.save_for_backward(gF, gr, gp)
            return loss.reshape(())

        @staticmethod
        def backward(ctx, gout):
            gF, gr, gp = ctx.saved_tensors
            return gout * gF, gout * gr, gout * gp, None, None

    return MorseLoss, EamLoss


def morse_loss(params, fm: ForceMatch):
    return _autograd()[0].apply(params, fm)


def eam_loss(F, rho, phi, fm: ForceMatch, tables: dict):
    return _autograd()[1].apply(F, rho, phi, fm, tables)


def adam_fit(loss_fn, params: list, steps: int = 200, lr: float = 1e-3,
             lr_final: float | None = None):
    """Runs `steps` Adam steps on loss_fn(*params); returns (losses, seconds)
    with the time measured by CUDA events around the loop.  lr_final: the
    step size decays from lr to lr_final on a cosine (constant without)."""
    import math

    import torch
    opt = torch.optim.Adam(params, lr=lr)
    losses = torch.zeros(steps, dtype=torch.float64, device=params[0].device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for k in range(steps):
        if lr_final is not None:
            c = 0.5 * (1.0 + math.cos(math.pi * k / max(1, steps - 1)))
            for grp in opt.param_groups:
                grp["lr"] = lr_final + (lr - lr_final) * c
        opt.zero_grad(set_to_none=True)
        loss = loss_fn(*params)
        loss.backward()
        opt.step()
        losses[k] = loss.detach()
    end.record()
    torch.cuda.synchronize()
    return losses.cpu().numpy(), start.elapsed_time(end) * 1e-3


def eam_table_meta(eam) -> dict:
    """ntypes / nrho / drho / nr / dr of an EamAlloy (api.EamAlloy)."""
    inf = eam.info()
    return {k: inf[k] for k in ("ntypes", "nrho", "drho", "nr", "dr")}


def eam_coeff_tensors(eam, device="cuda"):
    """(F, rho, phi) packed coefficient tensors of an EamAlloy."""
    import torch
    inf = eam.info()
    nt = inf["ntypes"]
    F = np.stack([eam.coeffs(0, t) for t in range(nt)])
    rho = np.stack([eam.coeffs(1, t) for t in range(nt)])
    phi = np.stack([eam.coeffs(2, p) for p in range(nt * (nt + 1) // 2)])
    return tuple(torch.as_tensor(a, dtype=torch.float64, device=device).contiguous()
                 for a in (F, rho, phi))


def eam_snapshots(eam, ncell=10, a=3.615, t=1200.0, nsnap=64, every=100, seed=77, dt=0.001):
    """Snapshots of an FP64 NVE run (FastPipelineScheduler, this library):
    ncell^3 FCC cells at temperature t, one snapshot every `every` steps.
    Returns (positions[nsnap, n, 3], types[n], lo, hi)."""
    from .api import FastPipelineScheduler, make_config
    from .workloads import fcc_system
    s = fcc_system(ncell, a, t, seed)
    box = Box.make(s.lo, s.hi)
    sc = FastPipelineScheduler(box, s.n, eam, make_config(dt=dt, r_skin=0.3, rebuild_every=10,
                                                         precision="fp64"))
    sc.upload(s.positions, s.velocities, None, s.types, s.ids, s.masses)
    out = np.zeros((nsnap, s.n, 3), np.float64)
    t0 = time.perf_counter()
    for k in range(nsnap):
        sc.run_until((k + 1) * every)
        out[k] = sc.download().positions
    sc.close()
    _ = t0
    return out, s.types.copy(), s.lo, s.hi
