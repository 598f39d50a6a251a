"""A caller written by the reference, unchanged, on this library: the
reference's benchmark driver (benchmarks/phase1_baseline/
bench_pipeline_scheduler.cu) compiled against include/tdmd_b200.hpp through
an include-path shim (tests/dropin/include maps each reference header path
onto the C++ layer), in both precision builds, by `make -C oracle dropin`
where the reference tree is present (the binaries in oracle/_ref travel
with the tree).

The driver reads a LAMMPS data file (tdmd::io::read_lammps_data),
initialises velocities, builds a FastPipelineScheduler (Morse or EAM) or
its default TD zone PipelineScheduler, runs warm-up and measured run_until
windows and prints JSON with the scheduler's counters; the test checks that
JSON against the same run made through this library's Python API: atoms,
steps, ticks and kernel launches of the measured region."""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

STEPS, WARMUP, SKIN = 40, 10, 0.3


def _exe(precision):
    p = os.path.join(ROOT, "oracle", "_ref", f"bench_pipeline_scheduler_b200_{precision}")
    if not os.path.exists(p):
        pytest.skip("the reference driver was not built here (make -C oracle dropin)")
    return p


def _python_launches(sysm, potential, precision, setfl):
    from tdmd_claude_b200 import (Box, EamAlloy, FastPipelineScheduler, MorseParams,
                                  make_config)
    cfg = make_config(dt=0.001, r_skin=SKIN, rebuild_every=10, precision=precision)
    pot = EamAlloy().read_setfl(setfl) if potential == "eam" else \
        MorseParams.make(0.3429, 1.3588, 2.866, 6.0)
    s = FastPipelineScheduler(Box.make(sysm.lo, sysm.hi), sysm.n, pot, cfg)
    s.upload(sysm.positions, sysm.velocities, None, sysm.types, sysm.ids, sysm.masses)
    s.run_until(WARMUP)
    a = s.stats()
    s.run_until(WARMUP + STEPS)
    b = s.stats()
    s.close()
    return b.kernel_launches - a.kernel_launches, b.ticks - a.ticks


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("potential", ["morse", "eam"])
def test_reference_driver_runs_unchanged(cuda, tmp_path, mishin_setfl, precision, potential):
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    sysm = W.fcc_system(10, 3.615, 300.0, seed=12)
    data = str(tmp_path / "fcc4000.data")
    TIO.write_lammps_data(data, sysm)
    out = str(tmp_path / "bench.json")
    args = [_exe(precision), "--scheduler", "fast_pipeline", "--data", data, "--steps",
            str(STEPS), "--warmup", str(WARMUP), "--skin", str(SKIN), "--output", out]
    if potential == "eam":
        args += ["--potential", "eam", "--eam", mishin_setfl]
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    with open(out) as f:
        d = json.load(f)
    assert d["scheduler"] == "fast_pipeline" and d["potential"] == potential
    assert d["n_atoms"] == sysm.n and d["n_steps"] == STEPS and d["ticks"] == STEPS
    assert d["timesteps_per_s"] > 0
    launches, ticks = _python_launches(sysm, potential, precision, mishin_setfl)
    assert ticks == STEPS
    assert d["kernel_launches_total"] == launches


def test_reference_driver_default_zone_scheduler(cuda, tmp_path):
    """The driver's default scheduler, the TD zone PipelineScheduler, runs
    on this library's whole-system path: the reference's zone count for the
    box (max(3, floor(L_x / rc))), the measured steps, no zone dependency
    checks (all zones step together)."""
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    sysm = W.fcc_system(10, 3.615, 300.0, seed=3)
    data = str(tmp_path / "fcc4000.data")
    TIO.write_lammps_data(data, sysm)
    out = str(tmp_path / "bench.json")
    r = subprocess.run([_exe("fp64"), "--data", data, "--steps", str(STEPS), "--warmup",
                        str(WARMUP), "--skin", str(SKIN), "--output", out],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    with open(out) as f:
        d = json.load(f)
    L = sysm.hi[0] - sysm.lo[0]
    assert d["n_zones"] == max(3, int(np.floor(L / 6.0)))
    assert d["n_atoms"] == sysm.n and d["n_steps"] == STEPS
    assert d["dep_check_calls"] == 0 and d["dep_check_failures"] == 0
    assert d["timesteps_per_s"] > 0
