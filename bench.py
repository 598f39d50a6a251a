"""Throughput of the TDMD force + integration path on B200.

Workload: 32x32x32 Cu FCC = 131,072 atoms (a = 3.615 A, +-0.01 A seeded
jitter, 300 K Maxwell-Boltzmann), analytic EAM tabulated as setfl splines
(Nr = Nrho = 2000, smoothly cut over 4.5-5.0 A), dt = 1 fs, skin 0.3 A,
neighbor rebuild every 10 steps, NVE -- mixed precision is the headline,
the plain FP64 path is measured in the same run.

One bench step = one FastPipelineScheduler::run_until window of 10 MD steps
(one neighbor rebuild + 10 force evaluations), i.e. 1,310,720 atom-steps.
L2 is flushed (256 MiB write) before every bench step, outside its timing.

  value     atom-steps/s, device time (CUDA events on the scheduler's stream
            around each window), inputs resident in HBM
  e2e       same metric through the C ABI with host buffers: upload (pinned
            host -> device) + run_until(10) + download (device -> pinned host)
            per step, wall clock
  roofline  dominant kernel (EAM force pass, mixed) vs the measured HBM copy
            bandwidth, algorithmic bytes from the gather model
  cpu_baseline  the reference's CPU path (oracle/_ref, compiled from its
            sources; else the oracle port), 1 thread, a bounded sample

`--impl reference` runs only the reference CPU path on the same workload.
Multi-GPU (torchrun): replicas only -- every rank runs its own system, the
value is the sum over ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WINDOW = 10            # MD steps per bench step (= rebuild interval)
NCELL = 32             # 32^3 FCC cells = 131,072 atoms
SKIN = 0.3
DT = 0.001
METRIC = "atom-steps/s (EAM 131k atoms) mixed vs FP64 on 1 B200 at force rel err <=1e-5"


# ---------------------------------------------------------------------------
def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and throttle reasons sampled during the timed region: every
    10 ms through NVML, or every 200 ms through nvidia-smi where NVML is
    unavailable."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []      # (sm_mhz, max_mhz, reasons bitmask)
        self.stop_flag = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = "GPU-" + str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _poll_nvml(self):
        nv, h = self.nvml
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop_flag.is_set():
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                     nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM),
                                     int(get_reasons(h))))
            except Exception:
                pass
            self.stop_flag.wait(0.01)

    def start(self):
        try:
            self.nvml = self._nvml_handle()
            self.t = threading.Thread(target=self._poll_nvml, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_flag.set()
            self.t.join(timeout=2)
            # NVML reason bits: sw power cap 0x4, hw slowdown 0x8,
            # sw thermal 0x20, hw thermal 0x40.
            bits = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                    "hw_thermal_slowdown": 0x40}
            if not self.samples:
                return None
            reasons = sorted({nm for nm, b in bits.items()
                              for _, _, r in self.samples if r & b})
            return {"sm_mhz": float(np.median([x[0] for x in self.samples])),
                    "sm_max_mhz": float(max(x[1] for x in self.samples)), "reasons": reasons,
                    "samples": len(self.samples), "source": "nvml, 10 ms"}
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], 0.0, set()
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = max(smax, float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 200 ms"}


# ---------------------------------------------------------------------------
def workload(seed=4321):
    from tdmd_claude_b200 import workloads as W
    return W.fcc_system(NCELL, 3.615, 300.0, seed), W.cu_eam_tables()


def make_eam(t):
    from tdmd_claude_b200 import EamAlloy
    return EamAlloy.from_tables(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)


def make_sched(sysm, eam, precision, **kw):
    from tdmd_claude_b200 import Box, FastPipelineScheduler, make_config
    s = FastPipelineScheduler(Box.make(sysm.lo, sysm.hi), sysm.n, eam,
                              make_config(dt=DT, r_skin=SKIN, rebuild_every=WINDOW,
                                          precision=precision, **kw))
    s.upload(sysm.positions, sysm.velocities, None, sysm.types, sysm.ids, sysm.masses)
    return s


def mean_neighbors(sysm, cutoff):
    """Mean full-list length K of the built list (for the roofline bytes)."""
    import torch

    from tdmd_claude_b200 import Box, DeviceNeighborList
    d = torch.as_tensor(sysm.positions, dtype=torch.float64, device="cuda")
    nl = DeviceNeighborList()
    nl.build(d, sysm.n, Box.make(sysm.lo, sysm.hi), cutoff, SKIN)
    c, _, _ = nl.host_csr()
    # interacting pairs (r < rc) for reference
    return float(c.mean())


def fcc_neighbors(a, r_list):
    """Sites of a perfect FCC lattice (constant a) within r_list of a site:
    the listed full-list length K the gather model counts."""
    m = int(np.ceil(2.0 * r_list / a)) + 1
    g = np.arange(-m, m + 1)
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    fcc = ((x + y + z) % 2) == 0          # FCC sites in units of a/2
    r2 = (x * x + y * y + z * z) * (0.5 * a) ** 2
    return int(np.count_nonzero(fcc & (r2 > 0) & (r2 < r_list * r_list)))


def cell_occupancy(n, L, r_list):
    """Atoms per cell of the reference grid, nc = max(3, floor(L / r_list))."""
    nc = max(3, int(np.floor(L / r_list)))
    return n / nc ** 3


def path_roofline(value, pot, precision, K, n_cell, hbm_gbs, R=None):
    """Whole-step gather model (bytes per atom-step) and the fraction of the
    measured HBM bandwidth it implies at `value` atom-steps/s.  Per atom-step:
    EAM FP64 224 + 64K, mixed 228 + 44K; Morse FP64 168 + 28K, mixed
    152 + 20K; plus the list build amortised over R steps,
    (27 n_cell (s_pos + 4) + 4K + 24) / R with s_pos = 24 (FP64) / 16 (mixed).
    Every neighbor access counts once (no cache reuse); spline tables are
    cache-resident."""
    R = R or WINDOW
    mixed = precision == "mixed"
    if pot == "eam":
        base = 228 + 44 * K if mixed else 224 + 64 * K
    else:
        base = 152 + 20 * K if mixed else 168 + 28 * K
    s_pos = 16 if mixed else 24
    b = base + (27 * n_cell * (s_pos + 4) + 4 * K + 24) / R
    ach = value * b / 1e9
    return {"bytes_per_atom_step": round(float(b), 1), "K": K, "atoms_per_cell": round(n_cell, 2),
            "achieved_gbs": ach, "frac": ach / hbm_gbs if hbm_gbs else None,
            "model": "gather model, whole step + list build / R"}


def shape_str(shapes):
    """{"density": "<lanes>x<batch>" or None, "force": ...} of an autotune result."""
    return {p: (f"{v[0]}x{v[1]}" if v else None) for p, v in shapes.items()}


def stats_shapes(st):
    """Launch shapes in use from a FastPipelineStats."""
    return shape_str({"density": (st.density_lanes_per_atom, st.density_nbr_batch)
                      if st.density_lanes_per_atom > 0 else None,
                      "force": (st.lanes_per_atom, st.nbr_batch)})


def timed_windows(sched, steps, warmup, flush, torch, dist=None):
    """Device ms per window (L2 flushed before each), max over ranks."""
    stream = torch.cuda.ExternalStream(sched.stream())
    step = sched.current_step()
    for _ in range(warmup):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        step += WINDOW
        sched.run_until(step)
    l0 = sched.stats().kernel_launches
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ms = []
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(k & 0xFF)
        step += WINDOW
        sched.run_until(step)
        ms.append(sched.last_window_ms())
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    wall = time.perf_counter() - t0
    launches = sched.stats().kernel_launches - l0
    from tdmd_claude_b200.replicas import max_over_ranks
    total = max_over_ranks(float(np.sum(ms)), dist, "cuda")
    return total, wall, launches, ms


def e2e_windows(sysm, eam, steps, warmup, torch, dist=None):
    """upload (pinned host) + run_until(WINDOW) + download (pinned host), wall
    (a barrier on both sides of the timed steps under a process group)."""
    from tdmd_claude_b200 import Box, FastPipelineScheduler, make_config
    s = FastPipelineScheduler(Box.make(sysm.lo, sysm.hi), sysm.n, eam,
                              make_config(dt=DT, r_skin=SKIN, rebuild_every=WINDOW,
                                          precision="mixed"))
    n = sysm.n
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    h_pos, h_vel = pin(sysm.positions), pin(sysm.velocities)
    h_typ, h_ids, h_m = pin(sysm.types), pin(sysm.ids), pin(sysm.masses)
    o_pos = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    o_vel = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    o_frc = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    h2d = h_pos.nbytes + h_vel.nbytes + h_typ.nbytes + h_ids.nbytes + h_m.nbytes
    d2h = o_pos.nbytes + o_vel.nbytes + o_frc.nbytes

    def one():
        s.upload_ptrs(h_pos.data_ptr(), h_vel.data_ptr(), 0, h_typ.data_ptr(), h_ids.data_ptr(),
                      h_m.data_ptr(), sysm.masses.size)
        s.run_until(WINDOW)
        s.download_ptrs(o_pos.data_ptr(), o_vel.data_ptr(), o_frc.data_ptr())

    for _ in range(warmup):
        one()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    if dist is not None:
        dist.barrier()
    s.close()
    return wall, h2d, d2h


def cpu_baseline_sample(sysm, t, nsteps):
    """The reference CPU path (or the oracle port) on the same system, 1 thread."""
    from oracle import oracle as O
    pos = sysm.positions.copy()
    vel = sysm.velocities.copy()
    frc = np.zeros_like(pos)
    lo, hi = np.array(sysm.lo), np.array(sysm.hi)
    R = O.ref()
    if R is not None:
        from tdmd_claude_b200 import io as TIO
        with tempfile.TemporaryDirectory() as d:
            p = os.path.join(d, "cu.eam.alloy")
            TIO.write_setfl(p, t)
            h = R.ref_eam_load(p.encode())
            import ctypes as C
            pe = C.c_double()
            sec = R.ref_run_cpu(h, 0, 0, 0, 0, pos.reshape(-1), vel.reshape(-1), frc.reshape(-1),
                                sysm.types, sysm.masses, 1, sysm.n, lo, hi, np.ones(3, np.int32),
                                DT, SKIN, WINDOW, nsteps, C.byref(pe))
            R.ref_eam_free(h)
        kind = "reference"
    else:
        oe = O.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
        t0 = time.perf_counter()
        O.md_run(pos, vel, sysm.types, sysm.masses, sysm.lo, sysm.hi, DT, SKIN, WINDOW, [nsteps],
                 eam=oe)
        sec = time.perf_counter() - t0
        kind = "port"
    return sec, kind


def host_cores(cap=64):
    """Host cores this process may use: its CPU affinity, bounded by a
    cgroup CPU quota where one is set, at most `cap`."""
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        with open("/sys/fs/cgroup/cpu.max") as f:
            quota, period = f.read().split()[:2]
        if quota != "max":
            n = min(n, max(1, int(int(quota) // int(period))))
    except (OSError, ValueError):
        pass
    return max(1, min(n, cap))


_CPU_BARRIER = None


def _cpu_worker_init(barrier):
    global _CPU_BARRIER
    _CPU_BARRIER = barrier
    os.environ["OMP_NUM_THREADS"] = "1"


def _cpu_worker(nsteps):
    """One process of the multi-core CPU baseline: the workload's system
    rebuilt here (same seed), then, once every worker is ready, the
    reference CPU loop (or the oracle port) for nsteps MD steps."""
    sysm, t = workload()
    _CPU_BARRIER.wait()
    return cpu_baseline_sample(sysm, t, nsteps)


def cpu_baseline_parallel(nsteps, cores):
    """The reference's CPU path is single-threaded; to use every host core
    it runs as `cores` independent processes, each advancing its own copy
    of the 131,072-atom system by nsteps, started together behind a
    barrier (processes spawned, never forked).  Returns (atom-steps/s of
    the whole job = cores * n * nsteps / the slowest process's loop time,
    that slowest time, the per-process times, kind)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(cores)
    with ctx.Pool(cores, initializer=_cpu_worker_init, initargs=(barrier,)) as pool:
        res = pool.map(_cpu_worker, [nsteps] * cores, chunksize=1)
    secs = [r[0] for r in res]
    n = NCELL ** 3 * 4
    return cores * n * nsteps / max(secs), max(secs), secs, res[0][1]


def nve_drift(sysm, eam, precision, nsteps, every=100):
    """Total-energy drift of an NVE run from the device energy log:
    least-squares slope of E_total/N against time (eV/atom/ns) and the
    largest |E_total - E_0|/N."""
    s = make_sched(sysm, eam, precision, energy_every=every,
                   energy_log_capacity=nsteps // every + 1)
    s.run_until(nsteps)
    log = s.energy_log()
    s.close()
    t_ns = log[:, 0] * DT * 1e-3
    e = (log[:, 1] + log[:, 2]) / sysm.n
    slope = float(np.polyfit(t_ns, e, 1)[0]) if len(e) > 1 else None
    return {"steps": nsteps, "ns": nsteps * DT * 1e-3, "slope_ev_per_atom_per_ns": slope,
            "max_abs_dev_ev_per_atom": float(np.abs(e - e[0]).max()) if len(e) else None}


def batch_bench(steps, warmup, flush, torch, precision="mixed", dist=None, rank=0, world=1,
                lanes=None, nbr_batch=None):
    """Batched replicas: 512 independent Cu FCC Morse systems (n^3 cells,
    n uniform 4..16, 100-1500 K), NVE, K = 10 steps per graph-replayed
    window; aggregate atom-steps/s and per-replica energy drift."""
    from tdmd_claude_b200 import Box, MorseParams, ReplicaBatch, make_config
    from tdmd_claude_b200 import workloads as W
    from tdmd_claude_b200.replicas import lpt_partition, sum_over_ranks
    systems = W.replica_set(512)
    if world > 1:  # whole replicas per rank, balanced by atom count
        mine = lpt_partition([s.n for s in systems], world)[rank]
        systems = [systems[i] for i in mine]
    b = ReplicaBatch([Box.make(s.lo, s.hi) for s in systems], [s.n for s in systems],
                     MorseParams.make(*W.MORSE_CU),
                     make_config(dt=DT, r_skin=SKIN, rebuild_every=WINDOW, precision=precision,
                                 energy_every=WINDOW, energy_log_capacity=steps + warmup + 8,
                                 **({"lanes_per_atom": lanes} if lanes else {}),
                                 **({"nbr_batch": nbr_batch} if nbr_batch else {})))
    b.upload(np.concatenate([s.positions for s in systems]),
             np.concatenate([s.velocities for s in systems]),
             np.concatenate([s.types for s in systems]), systems[0].masses)
    b.run_until(0)
    ms, _, launches, _ = timed_windows(b, steps, warmup, flush, torch, dist)
    steps_log, pk = b.energy_log()
    info = b.info()
    info["launch_shapes"] = stats_shapes(b.stats())
    natoms = np.array([s.n for s in systems], np.float64)
    etot = (pk[:, :, 0] + pk[:, :, 1]) / natoms          # eV/atom per window
    t_ns = steps_log * DT * 1e-3
    slopes = np.polyfit(t_ns, etot, 1)[0] if len(t_ns) > 1 else np.zeros(len(systems))
    b.close()
    atoms = sum_over_ranks(info["natoms"], dist, "cuda")
    slopes = np.atleast_1d(slopes)
    value = atoms * WINDOW * steps / (ms * 1e-3)
    hbm, _ = measured_peaks()
    K = fcc_neighbors(3.615, W.MORSE_CU[3] + SKIN)
    occ = float(np.sum([s.n * cell_occupancy(s.n, s.hi[0] - s.lo[0], W.MORSE_CU[3] + SKIN)
                        for s in systems]) / np.sum([s.n for s in systems]))
    return {"value": value, "unit": "atom-steps/s", "ms_per_window": ms / steps,
            "timesteps_per_s_each_replica": WINDOW * steps / (ms * 1e-3),
            "path_roofline": path_roofline(value, "morse", precision, K, occ, hbm),
            "replicas": 512, "atoms": int(atoms), "ranks": world, "precision": precision,
            "launch_shapes": info["launch_shapes"],
            "kernel_launches_timed": launches,
            "drift_ev_per_atom_per_ns": {"median_abs": float(np.median(np.abs(slopes))),
                                         "max_abs": float(np.max(np.abs(slopes))),
                                         "over_ps": float(t_ns[-1] - t_ns[0]) * 1e3
                                         if len(t_ns) > 1 else 0.0},
            "workload": "512 Cu FCC Morse replicas, n^3 cells n~U{4..16}, T~U(100,1500) K, "
                        "rc 6.0 skin 0.3, K=10 steps per graph",
            "_slopes": slopes}


def morse256_bench(torch, nsteps=1000):
    """The reference's CPU-runnable case: 4^3 Cu FCC (256 atoms), Morse
    rc 6.0, skin 0.3, 300 K, NVE dt 1 fs, nsteps steps in windows of 10 (a
    few microseconds of work per step: launch and graph-replay latency
    bound).  timesteps/s from the device time of the windows, and the energy
    drift of the run from the device energy log."""
    from tdmd_claude_b200 import Box, FastPipelineScheduler, MorseParams, make_config
    from tdmd_claude_b200 import workloads as W
    sysm = W.fcc_system(4, 3.615, 300.0, 4321)
    out = {}
    for prec in ("mixed", "fp64"):
        s = FastPipelineScheduler(Box.make(sysm.lo, sysm.hi), sysm.n,
                                  MorseParams.make(*W.MORSE_CU),
                                  make_config(dt=DT, r_skin=SKIN, rebuild_every=WINDOW,
                                              precision=prec, energy_every=WINDOW,
                                              energy_log_capacity=nsteps // WINDOW + 1))
        s.upload(sysm.positions, sysm.velocities, None, sysm.types, sysm.ids, sysm.masses)
        s.run_until(0)
        for w in range(3):                  # warm-up windows (graphs captured)
            s.run_until((w + 1) * WINDOW)
        s.upload(sysm.positions, sysm.velocities, None, sysm.types, sysm.ids, sysm.masses)
        s.run_until(0)
        ms = 0.0
        for w in range(nsteps // WINDOW):
            s.run_until((w + 1) * WINDOW)
            ms += s.last_window_ms()
        log = s.energy_log()
        s.close()
        t_ns = log[:, 0] * DT * 1e-3
        e = (log[:, 1] + log[:, 2]) / sysm.n
        out[prec] = {"timesteps_per_s": nsteps / (ms * 1e-3),
                     "atom_steps_per_s": sysm.n * nsteps / (ms * 1e-3),
                     "drift_ev_per_atom_per_ns": float(np.polyfit(t_ns, e, 1)[0]),
                     "steps": nsteps}
    out["workload"] = ("Cu FCC 4^3 cells = 256 atoms, Morse (0.3429, 1.3588, 2.866, rc 6.0), "
                       "skin 0.3, 300 K, NVE dt 1 fs, energy log every 10 steps")
    return out


def td_ring_bench(torch, ncell=32, steps=30):
    """The TD zone ring (DistributedPipelineScheduler) on one rank: 32^3 Cu
    FCC (131 072 atoms), Morse rc 6.0, skin 0.3, 300 K, FP64, windows of 10
    steps, host wall clock around synchronised run_until calls (its steps are
    orchestrated from the host: one kick-drift, one force call per zone and
    one closing kick per step); beside it the library's FastPipelineScheduler
    on the same system and schedule, device time.  Both the same state at the
    end (max position difference reported)."""
    from tdmd_claude_b200 import Box, FastPipelineScheduler, MorseParams, make_config
    from tdmd_claude_b200 import workloads as W
    from tdmd_claude_b200.distributed import DistributedConfig, DistributedPipelineScheduler
    sysm = W.fcc_system(ncell, 3.615, 300.0, 4321)
    box, mp_ = Box.make(sysm.lo, sysm.hi), MorseParams.make(*W.MORSE_CU)
    ring = DistributedPipelineScheduler(box, sysm.n, mp_, DistributedConfig(
        dt=DT, r_skin=SKIN, rebuild_every=WINDOW))
    ring.upload(sysm.positions, sysm.velocities, None, sysm.types, sysm.ids, sysm.masses)
    ring.run_until(WINDOW)                   # warm-up window
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ring.run_until(WINDOW + steps)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    fast = FastPipelineScheduler(box, sysm.n, mp_, make_config(
        dt=DT, r_skin=SKIN, rebuild_every=WINDOW, precision="fp64"))
    fast.upload(sysm.positions, sysm.velocities, None, sysm.types, sysm.ids, sysm.masses)
    fast.run_until(WINDOW)
    ms = 0.0
    for w in range(steps // WINDOW):
        fast.run_until(WINDOW * (w + 2))
        ms += fast.last_window_ms()
    p, _, _, _, ids = ring.download()
    q = fast.download().positions
    L = np.array(sysm.hi) - np.array(sysm.lo)
    d = p[np.argsort(ids)] - q
    d -= np.round(d / L) * L
    fast.close()
    return {"workload": f"Cu FCC {ncell}^3 cells = {sysm.n} atoms, Morse rc 6.0, skin 0.3, "
                        "300 K, FP64, rebuild every 10",
            "ranks": 1, "zones": ring.partition().n_zones,
            "value": sysm.n * steps / wall, "unit": "atom-steps/s",
            "ms_per_step": 1e3 * wall / steps, "timing": "host wall clock",
            "fast_pipeline_value": sysm.n * steps / (ms * 1e-3),
            "max_abs_position_diff_vs_fast_pipeline": float(np.abs(d).max()),
            "note": "one rank; the ring exchange (NCCL) is unmeasured on one GPU"}


def ternary_bench(steps, warmup, flush, torch, total_steps=2000):
    """Equiatomic random ternary FCC alloy, 100^3 cells = 4,000,000 atoms
    (a = 3.56 A), per-species analytic EAM, mixed precision, NVT
    (Nose-Hoover chain 3, 1000 K, tau 0.1 ps), adaptive dt =
    clamp(0.05 rc / v_max, 0.1 fs, 2 fs)."""
    from tdmd_claude_b200 import workloads as W
    sysm = W.ternary(100, t_target=1000.0)
    t = W.ternary_eam_tables()
    eam = make_eam(t)
    s = make_sched(sysm, eam, "mixed", t_target=1000.0, t_period=0.1, nhc_length=3,
                   adaptive_dt=True, dt_min=0.0001, dt_max=0.002, c2=0.05)
    s.run_until(0)
    ms, _, launches, _ = timed_windows(s, steps, warmup, flush, torch, None)
    n_dof = 3 * sysm.n - 3
    dt, _, _ = s.thermostat_state()
    pe, ke, _ = s.energies()
    temp = 2.0 * ke / (n_dof * 8.617333262e-5)
    # The run starts from the lattice at 1000 K, so equipartition halves the
    # kinetic temperature within ~0.1 ps; the rest of the workload's 2 000
    # steps (untimed) shows the chain bringing it back to the target.
    s.run_until(total_steps)
    dt2, _, _ = s.thermostat_state()
    _, ke2, _ = s.energies()
    s.close()
    temp2 = 2.0 * ke2 / (n_dof * 8.617333262e-5)
    value = sysm.n * WINDOW * steps / (ms * 1e-3)
    hbm, _ = measured_peaks()
    rl = t.cutoff + SKIN
    return {"value": value, "unit": "atom-steps/s",
            "timesteps_per_s": WINDOW * steps / (ms * 1e-3),
            "path_roofline": path_roofline(value, "eam", "mixed", fcc_neighbors(3.56, rl),
                                           cell_occupancy(sysm.n, sysm.hi[0] - sysm.lo[0], rl),
                                           hbm),
            "ms_per_window": ms / steps, "atoms": sysm.n, "precision": "mixed",
            "kernel_launches_timed": launches, "dt_ps_at_end": dt, "temperature_K_at_end": temp,
            "after_total_steps": {"steps": total_steps, "dt_ps": dt2, "temperature_K": temp2},
            "workload": "ternary FCC alloy 100^3 cells (4,000,000 atoms), EAM 3 species, "
                        "NVT NHC-3 1000 K, adaptive dt"}


def size_scaling_bench(steps, warmup, flush, torch, ncells=(32, 64, 128, 160)):
    """The headline workload (Cu FCC, analytic EAM, skin 0.3, rebuild every
    10) at 4 n^3 atoms for each n in ncells, mixed and FP64, one system per
    GPU: atom-steps/s out of L2 (the 32^3 system's ~55 MB stays resident in
    the 126 MB L2; 128^3 and 160^3 hold 3-8 GB) and the device memory each
    scheduler holds."""
    from tdmd_claude_b200 import workloads as W
    t = W.cu_eam_tables()
    eam = make_eam(t)
    hbm, _ = measured_peaks()
    rl = t.cutoff + SKIN
    K = fcc_neighbors(3.615, rl)
    out = {}
    for nc in ncells:
        sysm = W.fcc_system(nc, 3.615, 300.0, 4321 + nc)
        row = {"atoms": sysm.n}
        for prec in ("mixed", "fp64"):
            torch.cuda.synchronize()
            free0, _ = torch.cuda.mem_get_info()
            s = make_sched(sysm, eam, prec)
            s.run_until(0)
            torch.cuda.synchronize()
            free1, _ = torch.cuda.mem_get_info()
            ms, _, _, _ = timed_windows(s, steps, warmup, flush, torch, None)
            st = s.stats()
            s.close()
            value = sysm.n * WINDOW * steps / (ms * 1e-3)
            row[prec] = {"value": value, "ms_per_window": ms / steps,
                         "device_bytes": int(free0 - free1),
                         "launch_shapes": stats_shapes(st),
                         "path_roofline": path_roofline(
                             value, "eam", prec, K,
                             cell_occupancy(sysm.n, sysm.hi[0] - sysm.lo[0], rl), hbm)}
        row["mixed_over_fp64"] = row["mixed"]["value"] / row["fp64"]["value"]
        out[f"{nc}^3"] = row
        del sysm
    return {"unit": "atom-steps/s", "sizes": out,
            "workload": "Cu FCC n^3 cells, analytic EAM, NVE, skin 0.3, rebuild every 10; "
                        "L2 flushed (256 MiB write) before every window"}


def fit_bench(torch, adam_steps=200, nsnap=64, continue_morse=True):
    """Force matching: nsnap snapshots of a 10^3-cell Cu FCC (4,000 atoms)
    FP64 NVE run at 1200 K (one every 100 steps, config-1 EAM); targets from
    the FP64 forces of parameters perturbed by seeded 5 % Gaussian noise;
    loss = mean squared force error.  Adjoint gradients (mixed precision,
    FP64 accumulation) for Morse (D, alpha, r0) and all EAM spline
    coefficients; Adam steps timed with CUDA events; the Morse adjoint is
    checked against central differences (h = 1e-6 relative) of the FP64
    loss."""
    from tdmd_claude_b200 import Box
    from tdmd_claude_b200 import fitting as FT
    from tdmd_claude_b200 import workloads as W
    rng = np.random.default_rng(4242)
    t = W.cu_eam_tables()
    eam = make_eam(t)
    pos, types, lo, hi = FT.eam_snapshots(eam, ncell=10, t=1200.0, nsnap=nsnap, every=100)
    box = Box.make(lo, hi)
    out = {"snapshots": nsnap, "atoms_per_snapshot": int(pos.shape[1]), "adam_steps": adam_steps}
    # Morse
    m0 = np.array(W.MORSE_CU[:3])
    true = m0 * (1.0 + 0.05 * rng.standard_normal(3))
    ref64 = FT.ForceMatch(pos, types, box, W.MORSE_CU[3], "fp64")
    tgt = ref64.morse_forces(true)
    ref64.set_targets(tgt)
    fm = FT.ForceMatch(pos, types, box, W.MORSE_CU[3], "mixed")
    fm.set_targets(tgt)

    def loss64(p):
        prm = torch.tensor(p, dtype=torch.float64, device="cuda")
        lo_ = torch.zeros(1, dtype=torch.float64, device="cuda")
        g = torch.zeros(3, dtype=torch.float64, device="cuda")
        ref64.morse(prm, lo_, g)
        return float(lo_.item()), g.cpu().numpy()

    _, g64 = loss64(m0)
    fd = []
    for k in range(3):
        h = 1e-6 * m0[k]
        up, dn = m0.copy(), m0.copy()
        up[k] += h
        dn[k] -= h
        fd.append((loss64(up)[0] - loss64(dn)[0]) / (2 * h))
    p = torch.tensor(m0, dtype=torch.float64, device="cuda", requires_grad=True)
    losses, sec = FT.adam_fit(lambda q: FT.morse_loss(q, fm), [p], steps=adam_steps, lr=5e-3)
    p200 = p.detach().cpu().numpy().tolist()
    # Net forces of a near-lattice constrain mostly the pair curvature at the
    # neighbor shells, which leaves a shallow D - r0 valley: an untimed
    # continuation with a decaying step size shows where the fit goes.
    more = 10 * adam_steps if continue_morse else 1
    l2, sec2 = FT.adam_fit(lambda q: FT.morse_loss(q, fm), [p], steps=more, lr=5e-3,
                           lr_final=1e-5)
    pt = torch.tensor(true, dtype=torch.float64, device="cuda")
    out["morse"] = {
        "ms_per_adam_step": 1e3 * sec / adam_steps, "loss_first": float(losses[0]),
        "loss_last": float(losses[-1]), "params_true": true.tolist(),
        "params_fit": p200, "params_start": m0.tolist(),
        "loss_at_true_params": float(FT.morse_loss(pt, fm).item()),
        "continued": {"adam_steps": more, "lr": "5e-3 -> 1e-5 cosine",
                      "loss_last": float(l2[-1]),
                      "params_fit": p.detach().cpu().numpy().tolist(),
                      "params_rel_err": (np.abs(p.detach().cpu().numpy() - true) /
                                         np.abs(true)).tolist(),
                      "ms_per_adam_step": 1e3 * sec2 / more},
        "adjoint_vs_central_fd_rel": [abs(fd[k] - g64[k]) / abs(g64[k]) for k in range(3)]}
    # EAM: perturbed analytic parameters -> targets; fit all coefficients.
    f = 1.0 + 0.05 * rng.standard_normal(4)
    tp = W.analytic_eam(beta_f=(5.0 * f[0],), A_phi=(0.6 * f[1],), E_F=(1.2 * f[2],),
                        beta_phi=8.0 * f[3])
    eam_p = make_eam(tp)
    meta = FT.eam_table_meta(eam_p)
    Fp, rp, pp = FT.eam_coeff_tensors(eam_p)
    fm.close()
    ref64.close()
    # the EAM tables end at their cutoff: lists and pairs use it
    ref64 = FT.ForceMatch(pos, types, box, t.cutoff, "fp64")
    fm = FT.ForceMatch(pos, types, box, t.cutoff, "mixed")
    tgt = ref64.eam_forces(meta, Fp, rp, pp)
    fm.set_targets(tgt)
    F, rho, phi = (x.clone().requires_grad_(True) for x in FT.eam_coeff_tensors(eam))
    losses, sec = FT.adam_fit(lambda a, b, c: FT.eam_loss(a, b, c, fm, meta), [F, rho, phi],
                              steps=adam_steps, lr=1e-4)
    out["eam"] = {"ms_per_adam_step": 1e3 * sec / adam_steps, "loss_first": float(losses[0]),
                  "loss_last": float(losses[-1]),
                  "coefficients": int(F.numel() + rho.numel() + phi.numel()),
                  "perturbation_factors": f.tolist()}
    fm.close()
    ref64.close()
    return out


def batch_eam_bench(steps, warmup, flush, torch, eam, precision, nrep=8):
    """nrep replicas of the headline system (32^3 Cu FCC cells, 131,072
    atoms each, own seeds) as one EAM batch: every pass is one launch over
    all nrep * 131,072 atoms; NVE, windows of 10 steps."""
    from tdmd_claude_b200 import Box, ReplicaBatch, make_config
    from tdmd_claude_b200 import workloads as W
    systems = [W.fcc_system(NCELL, 3.615, 300.0, 5000 + r) for r in range(nrep)]
    b = ReplicaBatch([Box.make(s.lo, s.hi) for s in systems], [s.n for s in systems], eam,
                     make_config(dt=DT, r_skin=SKIN, rebuild_every=WINDOW, precision=precision))
    b.upload(np.concatenate([s.positions for s in systems]),
             np.concatenate([s.velocities for s in systems]),
             np.concatenate([s.types for s in systems]), systems[0].masses)
    b.run_until(0)
    ms, _, launches, _ = timed_windows(b, steps, warmup, flush, torch, None)
    info = b.info()
    info["launch_shapes"] = stats_shapes(b.stats())
    b.close()
    value = info["natoms"] * WINDOW * steps / (ms * 1e-3)
    hbm, _ = measured_peaks()
    rl = eam.cutoff() + SKIN
    s0 = systems[0]
    return {"value": value, "unit": "atom-steps/s",
            "timesteps_per_s_each_replica": WINDOW * steps / (ms * 1e-3),
            "path_roofline": path_roofline(value, "eam", precision, fcc_neighbors(3.615, rl),
                                           cell_occupancy(s0.n, s0.hi[0] - s0.lo[0], rl), hbm),
            "ms_per_window": ms / steps, "replicas": nrep, "atoms": info["natoms"],
            "launch_shapes": info["launch_shapes"],
            "kernel_launches_timed": launches}


def batch_eam_drift(eam, precision, nsteps=10000, nrep=8, every=100):
    """Per-replica NVE energy drift of the nrep x 131,072-atom EAM batch:
    nsteps steps in windows of `every` (the energy log writes each replica's
    PE and KE at every window's end, on the device); least-squares slope of
    E_total/N against time per replica, eV/atom/ns.  Untimed."""
    from tdmd_claude_b200 import Box, ReplicaBatch, make_config
    from tdmd_claude_b200 import workloads as W
    systems = [W.fcc_system(NCELL, 3.615, 300.0, 5000 + r) for r in range(nrep)]
    b = ReplicaBatch([Box.make(s.lo, s.hi) for s in systems], [s.n for s in systems], eam,
                     make_config(dt=DT, r_skin=SKIN, rebuild_every=WINDOW, precision=precision,
                                 energy_every=every, energy_log_capacity=nsteps // every + 4))
    b.upload(np.concatenate([s.positions for s in systems]),
             np.concatenate([s.velocities for s in systems]),
             np.concatenate([s.types for s in systems]), systems[0].masses)
    b.run_until(0)
    for k in range(every, nsteps + 1, every):
        b.run_until(k)
    steps_log, pk = b.energy_log()
    b.close()
    natoms = np.array([s.n for s in systems], np.float64)
    etot = (pk[:, :, 0] + pk[:, :, 1]) / natoms
    t_ns = steps_log * DT * 1e-3
    slopes = np.atleast_1d(np.polyfit(t_ns, etot, 1)[0])
    return {"steps": nsteps, "ns": nsteps * DT * 1e-3, "replicas": nrep,
            "slope_ev_per_atom_per_ns": slopes.tolist(),
            "max_abs_slope": float(np.abs(slopes).max()),
            "max_abs_dev_ev_per_atom": float(np.abs(etot - etot[0]).max())}


def reference_gpu_sample(sysm, t, windows=50, warm=5, repeats=3):
    """The reference's own GPU FastPipelineScheduler (oracle/_ref, compiled
    from its sources, FP64 and mixed builds) on the same system: host wall
    clock around `windows` whole run_until windows (it synchronizes the host
    inside a rebuild), after `warm` untimed ones, repeated `repeats` times
    with a fresh scheduler each; median and range of the repeats.  None
    where those libraries or a GPU are absent."""
    import ctypes as C
    out = {}
    try:
        import torch
        if not torch.cuda.is_available():
            return None
    except Exception:
        return None
    from tdmd_claude_b200 import io as TIO
    for prec in ("fp64", "mixed"):
        path = os.path.join(ROOT, "oracle", "_ref", f"libtdmd_ref_gpu_{prec}.so")
        if not os.path.exists(path):
            continue
        L = C.CDLL(path)
        L.refgpu_run_eam.restype = C.c_double
        L.refgpu_last_error.restype = C.c_char_p
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
        L.refgpu_run_eam.argtypes = [C.c_char_p, f64p, f64p, i32p, f64p, C.c_int32, C.c_int32,
                                     f64p, f64p, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                     C.c_int32, C.c_int32]
        secs = []
        with tempfile.TemporaryDirectory() as d:
            setfl = os.path.join(d, "cu.eam.alloy")
            TIO.write_setfl(setfl, t)
            for _ in range(repeats):
                sec = L.refgpu_run_eam(setfl.encode(), np.ascontiguousarray(sysm.positions),
                                       np.ascontiguousarray(sysm.velocities),
                                       np.ascontiguousarray(sysm.types, dtype=np.int32),
                                       np.ascontiguousarray(sysm.masses), sysm.masses.size,
                                       sysm.n, np.array(sysm.lo, np.float64),
                                       np.array(sysm.hi, np.float64), DT, SKIN, WINDOW, WINDOW,
                                       warm, windows)
                if sec <= 0:
                    break
                secs.append(sec)
        if not secs:
            out[prec] = {"error": L.refgpu_last_error().decode()}
            continue
        vals = sorted(sysm.n * WINDOW * windows / x for x in secs)
        out[prec] = {"value": float(np.median(vals)), "min": vals[0], "max": vals[-1],
                     "samples": vals, "unit": "atom-steps/s",
                     "ms_per_window_median": float(np.median([1e3 * x / windows for x in secs])),
                     "windows_per_sample": windows, "warmup_windows": warm,
                     "timing": "host wall clock around run_until windows (median of "
                               f"{len(secs)} samples, fresh scheduler each)"}
    return out or None


# ---------------------------------------------------------------------------
def run_reference(args, rank, world):
    if rank != 0:
        return
    sysm, t = workload()
    warm = max(1, min(args.warmup, 2))
    cpu_baseline_sample(sysm, t, warm)          # warm caches/pages (untimed)
    cores = args.cpu_cores or host_cores()
    if cores > 1:
        value, sec, secs, kind = cpu_baseline_parallel(args.steps, cores)
    else:
        sec, kind = cpu_baseline_sample(sysm, t, args.steps)
        value, secs = sysm.n * args.steps / sec, [sec]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "atom-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sec / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "eam_cu_fcc_131072", "atoms": sysm.n, "precision": "fp64 (CPU)",
                   "dt_fs": 1.0, "skin": SKIN, "rebuild_every": WINDOW,
                   "step": "one MD timestep of every process's copy of the system",
                   "processes": cores,
                   "per_process_loop_s": secs},
        "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": cores, "kind": kind,
                         "sample": f"{args.steps} MD steps of the 131,072-atom EAM system in "
                                   f"each of {cores} concurrent single-threaded processes "
                                   "(the reference CPU loop has no threads; rebuild every 10); "
                                   "value = all processes' atom-steps / the slowest loop"},
        "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if not args.no_ref_gpu:
        # context only (the arm's value is the CPU reference): the reference's
        # own GPU FastPipelineScheduler on the same system and GPU
        line["reference_gpu_same_box"] = reference_gpu_sample(sysm, t)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=10, help="reference CPU sample size")
    ap.add_argument("--cpu-cores", type=int, default=0,
                    help="processes of the CPU baseline / reference arm (0: every usable host "
                         "core, at most 64)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--kernels-only", action="store_true",
                    help="only the mixed timed windows (for profiler captures); no JSON line")
    ap.add_argument("--case", default="eam-mixed",
                    choices=["eam-mixed", "eam-fp64", "eam-nvt-ev", "morse-batch",
                             "morse-batch-fp64", "fit", "ternary"],
                    help="workload of --kernels-only: the 131,072-atom EAM system (mixed, "
                         "FP64, or mixed NVT with energy/virial every step), the 512 "
                         "Morse replicas, force matching, or the 4M-atom ternary NVT run")
    ap.add_argument("--lanes", type=int, default=None,
                    help="lanes per atom for --kernels-only (EAM: default 4, no autotune; "
                         "Morse replicas: autotuned unless given)")
    ap.add_argument("--nbr-batch", type=int, default=None,
                    help="neighbors per lane sweep for --kernels-only (EAM: default 2, the "
                         "autotuner's usual choice at 131,072 atoms; Morse replicas: autotuned "
                         "unless given)")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip timing the reference's own GPU scheduler (same-run context)")
    ap.add_argument("--no-fit", action="store_true",
                    help="skip the force-matching (adjoint + Adam) figure")
    ap.add_argument("--no-ternary", action="store_true",
                    help="skip the 4M-atom ternary NVT + adaptive-dt figure")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched-replica (512 Morse systems) figure")
    ap.add_argument("--no-sizes", action="store_true",
                    help="skip the single-system size sweep (131 k to 16.4 M atoms)")
    ap.add_argument("--drift-steps", type=int, default=50000,
                    help="NVE steps for the energy-drift figure (0 = skip)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = env_rank()
    if world > 1:
        # N replicas: the headline, e2e and the sharded batch figure; the
        # single-GPU extras (drift, force matching, 4 M-atom ternary) are not
        # repeated per rank.
        args.no_fit = args.no_ternary = args.no_sizes = True
        args.drift_steps = 0
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as D
        D.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = D

    sysm, t = workload(seed=4321 + rank)
    eam = make_eam(t)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    if args.kernels_only:
        if args.case == "fit":
            fit_bench(torch, adam_steps=args.steps, nsnap=64, continue_morse=False)
        elif args.case == "ternary":
            ternary_bench(args.steps, args.warmup, flush, torch, total_steps=0)
        elif args.case.startswith("morse-batch"):
            prec = "fp64" if args.case.endswith("fp64") else "mixed"
            batch_bench(args.steps, args.warmup, flush, torch, prec, dist, rank, world,
                        args.lanes, args.nbr_batch)
        else:
            prec = "fp64" if args.case == "eam-fp64" else "mixed"
            kw = {}
            if args.case == "eam-nvt-ev":
                kw = dict(t_target=300.0, t_period=0.1, nhc_length=3, energy_every=1,
                          energy_log_capacity=16)
            s32 = make_sched(sysm, eam, prec, lanes_per_atom=args.lanes or 4,
                             nbr_batch=args.nbr_batch or 2, **kw)
            s32.run_until(0)
            timed_windows(s32, args.steps, args.warmup, flush, torch, dist)
            s32.close()
        if dist is not None:
            dist.destroy_process_group()
        return
    K = mean_neighbors(sysm, t.cutoff)

    # Force accuracy of the mixed path vs FP64 on the same state.
    s64 = make_sched(sysm, eam, "fp64")
    s32 = make_sched(sysm, eam, "mixed")
    s64.run_until(0)
    s32.run_until(0)
    shapes32, tune32 = s32.autotune()
    shapes64, tune64 = s64.autotune()
    f64 = s64.download().forces
    f32 = s32.download().forces.astype(np.float64)
    rel_err = float(np.sqrt(((f32 - f64) ** 2).sum() / (f64 ** 2).sum()))

    # Headline: mixed.
    clocks = ClockSampler(local)
    clocks.start()
    ms_mixed, wall_mixed, launches, per = timed_windows(s32, args.steps, args.warmup, flush, torch,
                                                        dist)
    clk = clocks.stop()
    # Plain FP64 path, same protocol.
    ms_fp64, wall_fp64, _, _ = timed_windows(s64, args.steps, args.warmup, flush, torch, dist)

    units = world * sysm.n * WINDOW * args.steps
    value = units / (ms_mixed * 1e-3)
    value64 = units / (ms_fp64 * 1e-3)

    # Per-kernel times: the same windows replayed from graphs of their own
    # with event-record nodes around each phase (L2 flushed before each); a
    # first window captures those graphs, then the counters start from zero.
    nprof = max(5, args.steps // 3)

    def phase_times(sched):
        sched.set_profiling(True)
        timed_windows(sched, 1, 0, flush, torch, None)
        sched.set_profiling(True)
        ms, _, _, _ = timed_windows(sched, nprof, 0, flush, torch, None)
        k = sched.kernel_times()
        sched.set_profiling(False)
        return ms, k

    prof_ms32, kt = phase_times(s32)
    prof_ms64, kt64 = phase_times(s64)
    phase_check = {
        p: {"window_ms": w / nprof, "phase_sum_ms_per_window":
            sum(ms * n for ms, n in k.values()) / nprof}
        for p, w, k in (("mixed", prof_ms32, kt), ("fp64", prof_ms64, kt64))}

    # NVT (Nose-Hoover chain 3, tau 0.1 ps, 300 K), same protocol.
    snvt = make_sched(sysm, eam, "mixed", t_target=300.0,
                      t_period=0.1, nhc_length=3)
    snvt.run_until(0)
    ms_nvt, _, _, _ = timed_windows(snvt, args.steps, args.warmup, flush, torch, dist)
    snvt.close()
    value_nvt = units / (ms_nvt * 1e-3)

    drift = None
    if args.drift_steps > 0:
        drift = {"mixed": nve_drift(sysm, eam, "mixed", args.drift_steps),
                 "fp64": nve_drift(sysm, eam, "fp64", args.drift_steps)}

    batch = None
    if not args.no_batch:
        batch = {p: batch_bench(args.steps, args.warmup, flush, torch, p, dist, rank, world)
                 for p in ("mixed", "fp64")}
        # The Morse pair term is truncated at rc without a shift (as the
        # reference's), so E_total jumps by U(rc) each time a pair crosses
        # rc: the per-replica drift above is that physics, alike in FP64.
        # The precision effect is the per-replica mixed - FP64 difference.
        dd = np.abs(batch["mixed"].pop("_slopes") - batch["fp64"].pop("_slopes"))
        batch["drift_mixed_minus_fp64_ev_per_atom_per_ns"] = {
            "median_abs": float(np.median(dd)), "max_abs": float(np.max(dd)),
            "note": "Morse truncated at rc without shift (reference form): E_total "
                    "jumps by U(rc) = -9.6 meV per pair crossing, so single-run drift "
                    "is physical; same seeds and windows in both precisions"}

    beam = None
    if not args.no_batch:
        beam = {p: batch_eam_bench(args.steps, args.warmup, flush, torch, eam, p)
                for p in ("mixed", "fp64")}
        beam["mixed_batched_over_plain_fp64"] = beam["mixed"]["value"] / value64
        beam["mixed_over_fp64_batched"] = beam["mixed"]["value"] / beam["fp64"]["value"]
        if args.drift_steps > 0:
            # the single system's 50 ps: a 10 ps fit is dominated by the
            # Verlet energy fluctuation (~3e-6 eV/atom), not by drift
            dr = {p: batch_eam_drift(eam, p, nsteps=args.drift_steps, nrep=4)
                  for p in ("mixed", "fp64")}
            dd = np.abs(np.array(dr["mixed"]["slope_ev_per_atom_per_ns"]) -
                        np.array(dr["fp64"]["slope_ev_per_atom_per_ns"]))
            dr["mixed_minus_fp64_max_abs"] = float(dd.max())
            beam["nve_drift"] = dr
    fitfig = None if args.no_fit else fit_bench(torch)
    small = None if args.no_batch else morse256_bench(torch)
    ring = None if (args.no_batch or world > 1) else td_ring_bench(torch)
    ternary = None if args.no_ternary else ternary_bench(max(3, args.steps // 3), 3, flush,
                                                           torch)
    sizes = None if args.no_sizes else size_scaling_bench(max(3, args.steps // 5), 3, flush,
                                                          torch)

    hbm, peak_kind = measured_peaks()
    occ = cell_occupancy(sysm.n, sysm.hi[0] - sysm.lo[0], eam.cutoff() + SKIN)
    # gather model of the mixed force pass, plus the next step's kick + drift
    # it carries on (WINDOW-1) of WINDOW launches (144 B per atom)
    force_bytes = sysm.n * (48 + 24 * K) + sysm.n * 144 * (WINDOW - 1) / WINDOW
    dens_bytes = sysm.n * (40 + 20 * K)
    force_ms = kt["force"][0]
    achieved = force_bytes / (force_ms * 1e-3) / 1e9 if force_ms > 0 else None
    # traffic is a recorded figure (an ncu capture of this kernel on this
    # workload, summarised in profiles/), not measured by this run
    traffic, traffic_src = None, None
    prof_json = os.path.join(ROOT, "profiles", "eam_force_mixed_131k.json")
    if os.path.exists(prof_json):
        with open(prof_json) as f:
            rec = json.load(f)
        traffic = rec.get("dram_bytes_per_launch")
        traffic_src = {"recorded": "profiles/eam_force_mixed_131k.json",
                       "captured": rec.get("captured"), "kernel": rec.get("kernel"),
                       "command": rec.get("command")}

    # e2e: every rank times its own steps; the job's time is the slowest rank's
    from tdmd_claude_b200.replicas import max_over_ranks
    e2e_steps = max(3, args.steps)
    e2e_wall, h2d, d2h = e2e_windows(sysm, eam, e2e_steps, max(3, args.warmup), torch, dist)
    e2e_wall = max_over_ranks(e2e_wall, dist, "cuda")
    e2e_value = world * sysm.n * WINDOW * e2e_steps / e2e_wall

    # Same-run context: the reference's own GPU scheduler on this system and
    # GPU (host wall clock, as it synchronizes inside rebuilds), against this
    # run's host-wall windows and e2e figure.
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_ref_gpu:
        ref_gpu = reference_gpu_sample(sysm, t)
        if ref_gpu:
            ours = {"mixed_host_wall": units / wall_mixed, "fp64_host_wall": units / wall_fp64,
                    "e2e": e2e_value}
            ratios = {}
            for prec in ("mixed", "fp64"):
                ref_v = (ref_gpu.get(prec) or {}).get("value")
                if ref_v:
                    ratios[f"ours_{prec}_host_wall_over_ref_{prec}"] = \
                        ours[f"{prec}_host_wall"] / ref_v
                    ratios[f"ours_e2e_over_ref_{prec}"] = e2e_value / ref_v
            ref_gpu = {"reference": ref_gpu, "ours_same_run": ours, "ratios_vs_median": ratios,
                       "note": "host wall includes the L2-flush writes between windows"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = args.cpu_cores or host_cores()
        sec1, kind = cpu_baseline_sample(sysm, t, args.cpu_steps)
        if cores > 1:
            value_c, _, _, kind = cpu_baseline_parallel(args.cpu_steps, cores)
        else:
            value_c = sysm.n * args.cpu_steps / sec1
        cpu = {"value": value_c, "unit": "atom-steps/s", "cores": cores, "kind": kind,
               "one_core": sysm.n * args.cpu_steps / sec1,
               "sample": f"{args.cpu_steps} MD steps (rebuild every 10) of the same 131,072-atom "
                         f"EAM system in each of {cores} concurrent single-threaded processes "
                         "(the reference CPU loop has no threads); one_core: one process alone"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_mixed / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {
                "workload": "eam_cu_fcc_131072", "atoms": sysm.n, "precision": "mixed",
                "potential": "analytic Cu EAM as setfl splines, Nr=Nrho=2000, cut 4.5-5.0 A",
                "dt_fs": 1.0, "skin": SKIN, "rebuild_every": WINDOW,
                "md_steps_per_bench_step": WINDOW, "parallelism": f"replicas x{world}",
                "l2": "flushed (256 MiB write) before every bench step, outside its timing",
                "mean_neighbors_K": K,
                "launch_shapes": {"mixed": shape_str(shapes32), "fp64": shape_str(shapes64),
                                  "autotune_ms_mixed": tune32, "autotune_ms_fp64": tune64,
                                  "keys": "<pass> <lanes per atom>x<neighbors per lane sweep>"},
                "timesteps_per_s": value / sysm.n,
                "path_roofline": path_roofline(value, "eam", "mixed", K, occ, hbm),
                "fp64": {"value": value64, "ms_per_step": ms_fp64 / args.steps,
                         "timesteps_per_s": value64 / sysm.n,
                         "path_roofline": path_roofline(value64, "eam", "fp64", K, occ, hbm)},
                "mixed_over_fp64": value / value64,
                "force_rel_rms_err_mixed_vs_fp64": rel_err,
                "nvt_mixed": {"value": value_nvt, "ms_per_step": ms_nvt / args.steps,
                              "thermostat": "Nose-Hoover chain 3, tau 0.1 ps, 300 K"},
                "nve_drift": drift,
                "batched_replicas": batch,
                "batched_eam_131k_x8": beam,
                "ternary_4m_nvt_adaptive": ternary,
                "single_system_sizes": sizes,
                "morse_256_nve_1000": small,
                "td_ring_morse_131k": ring,
                "force_matching": fitfig,
                "wall_s_timed_region": wall_mixed,
                "reference_gpu_same_run": ref_gpu,
            },
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                         "traffic_source": traffic_src,
                         "ms_source": "CUDA events recorded by event-record nodes "
                                      "around each force launch inside the replayed window "
                                      "graphs (profiling graphs: plain edges between their "
                                      "kernels), same system and L2 flush as value",
                         "phases_vs_window": phase_check,
                         "kernel": "k_eam_force<GeoQ> (mixed)", "peak_source": peak_kind,
                         "bytes_per_launch": force_bytes, "ms_per_launch": force_ms,
                         "model": "gather model n*(48+24K) B, K = mean full-list length, "
                                  "+ 144 B/atom kick-drift on 9 of 10 launches"},
            "kernel_ms": {"mixed": kt, "fp64": kt64,
                          "density_bytes_per_launch": dens_bytes},
            "e2e": {"value": e2e_value, "unit": "atom-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                    "timing": "wall clock over the steps (barriers on both sides)"},
            "gpu_launches": launches,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    for s in (s32, s64):
        s.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
