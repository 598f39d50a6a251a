"""GPU Morse and EAM forces/energies/virials vs the oracle (C ABI).

Tolerances: FP64 <= 1e-10 relative (forces normalised by the RMS force,
energies relative); mixed RMS force error <= 1e-5 relative, energies 1e-6."""
from __future__ import annotations

import os
import tempfile

import numpy as np
import pytest

from conftest import golden, rel_rms

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
MIXED_FORCE_TOL = 1e-5


def _dev(torch, a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _box(lo, hi):
    from tdmd_claude_b200 import Box
    return Box.make(lo, hi)


def _morse_gpu(torch, pos, lo, hi, morse, skin, precision):
    from tdmd_claude_b200 import DeviceNeighborList, MorseParams, compute_morse_gpu
    n = len(pos)
    box = _box(lo, hi)
    d = _dev(torch, pos, torch.float64)
    nl = DeviceNeighborList()
    nl.build(d, n, box, morse[3], skin)
    fdt = torch.float64 if precision == "fp64" else torch.float32
    f = torch.zeros((n, 3), dtype=fdt, device="cuda")
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    w = torch.zeros(6, dtype=torch.float64, device="cuda")
    compute_morse_gpu(d, f, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), n, box,
                      MorseParams.make(*morse), e, w, precision=precision)
    torch.cuda.synchronize()
    return f.double().cpu().numpy(), float(e.item()), w.cpu().numpy()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_morse_c0_vs_oracle(cuda, oracle, precision):
    g = golden("ref_morse_256.json")
    pos = np.array(g["positions"])
    f, e, w = _morse_gpu(cuda, pos, g["lo"], g["hi"], g["morse"], g["skin"], precision)
    pe, fo, wo = oracle.morse_forces(pos, g["lo"], g["hi"], *g["morse"], g["skin"])
    assert np.array_equal(fo, np.array(g["reference_forces"]))
    if precision == "fp64":
        assert rel_rms(f, fo) < FP64_TOL
        assert abs(e - pe) / abs(pe) < FP64_TOL
        assert np.abs(w - wo).max() / np.abs(wo).max() < FP64_TOL
    else:
        assert rel_rms(f, fo) < MIXED_FORCE_TOL
        assert abs(e - pe) / abs(pe) < 1e-6
        assert np.abs(w - wo).max() / np.abs(wo).max() < MIXED_FORCE_TOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_morse_run0_lammps(cuda, precision):
    """VerifyLab run0-force-match thresholds: max |dF| 1e-12 (FP64), 5e-5 (mixed)."""
    g = golden("run0_morse_256.json")
    f, e, _ = _morse_gpu(cuda, np.array(g["positions"]), g["lo"], g["hi"], g["morse"], g["skin"],
                         precision)
    tol = g["tolerance_fp64"] if precision == "fp64" else g["tolerance_mixed"]
    assert np.abs(f - np.array(g["lammps_forces"])).max() < tol
    assert abs(e - g["reference_pe"]) / abs(g["reference_pe"]) < (1e-12 if precision == "fp64"
                                                                 else 1e-6)


def test_two_atoms_morse(cuda):
    g = golden("two_atoms_morse.json")
    p = g["potential"]
    pos = np.array([a["pos_A"] for a in g["atoms"]]) + 10.0
    f, e, _ = _morse_gpu(cuda, pos, (0, 0, 0), (30, 30, 30),
                         (p["D0_eV"], p["alpha_inv_A"], p["r0_A"], p["cutoff_A"]), 0.0, "fp64")
    assert abs(e - g["step0"]["U_eV"]) < 1e-14
    f1 = np.array(g["step0"]["force_on_atom_1_eV_per_A"])
    assert np.abs(f[0] - f1).max() / abs(f1[0]) < 1e-14
    f, e, _ = _morse_gpu(cuda, pos, (0, 0, 0), (30, 30, 30),
                         (p["D0_eV"], p["alpha_inv_A"], p["r0_A"], p["cutoff_A"]), 0.0, "mixed")
    assert np.abs(f[0] - f1).max() / abs(f1[0]) < 1e-6
    assert abs(e - g["step0"]["U_eV"]) < 1e-6


def _eam_gpu(torch, eam, pos, types, lo, hi, skin, precision):
    from tdmd_claude_b200 import DeviceEam, DeviceNeighborList
    n = len(pos)
    box = _box(lo, hi)
    d = _dev(torch, pos, torch.float64)
    t = _dev(torch, types, torch.int32)
    nl = DeviceNeighborList()
    nl.build(d, n, box, eam.cutoff(), skin)
    de = DeviceEam()
    de.upload_tables(eam)
    fdt = torch.float64 if precision == "fp64" else torch.float32
    f = torch.zeros((n, 3), dtype=fdt, device="cuda")
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    w = torch.zeros(6, dtype=torch.float64, device="cuda")
    rho = torch.zeros(n, dtype=torch.float64, device="cuda")
    fp = torch.zeros(n, dtype=torch.float64, device="cuda")
    de.compute(d, f, t, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), n, box, e, w, rho, fp,
               precision=precision)
    torch.cuda.synchronize()
    return (f.double().cpu().numpy(), float(e.item()), w.cpu().numpy(), rho.cpu().numpy(),
            fp.cpu().numpy())


def _analytic_eam(tables):
    from tdmd_claude_b200 import EamAlloy
    return EamAlloy.from_tables(tables.ntypes, tables.nrho, tables.drho, tables.nr, tables.dr,
                                tables.cutoff, tables.F, tables.rho, tables.rphi)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_eam_analytic_vs_oracle(cuda, oracle, precision):
    from tdmd_claude_b200 import workloads as W
    g = golden("ref_eam_256.json")
    m = golden("ref_morse_256.json")
    t = W.cu_eam_tables()
    eam = _analytic_eam(t)
    pos = np.array(m["positions"])
    types = np.ones(len(pos), np.int32)
    f, e, w, rho, fp = _eam_gpu(cuda, eam, pos, types, m["lo"], m["hi"], g["skin"], precision)
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    r = oe.forces(pos, types, m["lo"], m["hi"], g["skin"])
    assert r["pe"] == g["reference_pe"]
    if precision == "fp64":
        assert rel_rms(f, r["forces"]) < FP64_TOL
        assert abs(e - r["pe"]) / abs(r["pe"]) < FP64_TOL
        assert np.abs(rho - r["rho"]).max() / r["rho"].max() < FP64_TOL
        assert np.abs(fp - r["fp"]).max() / np.abs(r["fp"]).max() < FP64_TOL
        assert np.abs(w - r["virial"]).max() / np.abs(r["virial"]).max() < FP64_TOL
    else:
        assert rel_rms(f, r["forces"]) < MIXED_FORCE_TOL
        assert abs(e - r["pe"]) / abs(r["pe"]) < 1e-6
        assert np.abs(rho - r["rho"]).max() / r["rho"].max() < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_eam_ternary_vs_oracle(cuda, oracle, precision):
    """Three species: type-pair spline indexing (phi_index) and per-type
    density/embedding."""
    from tdmd_claude_b200 import workloads as W
    t = W.ternary_eam_tables()
    s = W.ternary(6, seed=3)
    eam = _analytic_eam(t)
    f, e, w, rho, fp = _eam_gpu(cuda, eam, s.positions, s.types, s.lo, s.hi, 0.3, precision)
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    r = oe.forces(s.positions, s.types, s.lo, s.hi, 0.3)
    tol = FP64_TOL if precision == "fp64" else MIXED_FORCE_TOL
    assert rel_rms(f, r["forces"]) < tol
    assert abs(e - r["pe"]) / abs(r["pe"]) < (FP64_TOL if precision == "fp64" else 1e-6)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_eam_setfl_reader_matches_oracle(cuda, oracle, precision):
    """The library's setfl reader + spline build equal the oracle's."""
    from tdmd_claude_b200 import EamAlloy
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    t = W.cu_eam_tables()
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "cu.eam.alloy")
        TIO.write_setfl(p, t)
        eam = EamAlloy().read_setfl(p)
        oe = oracle.OracleEam.from_setfl(p)
    for kind in (0, 1, 2):
        assert np.array_equal(eam.coeffs(kind, 0), oe.coeffs(kind, 0))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_eam_mishin_run0_lammps(cuda, mishin_setfl, precision):
    from tdmd_claude_b200 import EamAlloy
    g = golden("run0_eam_256.json")
    m = golden("run0_morse_256.json")
    eam = EamAlloy().read_setfl(mishin_setfl)
    pos = np.array(m["positions"])
    f, e, *_ = _eam_gpu(cuda, eam, pos, np.ones(256, np.int32), m["lo"], m["hi"], g["skin"],
                        precision)
    tol = g["tolerance_fp64"] if precision == "fp64" else g["tolerance_mixed"]
    assert np.abs(f - np.array(g["lammps_forces"])).max() < tol


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_stream_order_after_caller_kernels(cuda, oracle, precision):
    """Library kernels are launched with programmatic dependent launch: on a
    caller's stream they wait for the caller's preceding kernels.  Each round
    the caller zeroes the position buffer, runs a 128 MiB reduction and only
    then writes the positions, all on one stream, right before the list
    build and the force call (a library kernel that ran early would see
    every atom at the origin); the forces equal the oracle's every round."""
    torch = cuda
    from tdmd_claude_b200 import DeviceNeighborList, MorseParams, compute_morse_gpu
    g = golden("ref_morse_256.json")
    pos0 = np.array(g["positions"])
    n = len(pos0)
    box = _box(g["lo"], g["hi"])
    _, fo, _ = oracle.morse_forces(pos0, g["lo"], g["hi"], *g["morse"], g["skin"])
    s = torch.cuda.Stream()
    big = torch.rand(1 << 24, device="cuda", dtype=torch.float64)
    base = torch.tensor(pos0, device="cuda", dtype=torch.float64)
    d = torch.empty_like(base)
    fdt = torch.float64 if precision == "fp64" else torch.float32
    nl = DeviceNeighborList()
    torch.cuda.synchronize()
    for _ in range(4):
        with torch.cuda.stream(s):
            f = torch.zeros((n, 3), dtype=fdt, device="cuda")
            d.zero_()
            zero = (big * 0.0).sum()
            torch.add(base, zero, out=d)  # the kernel right before the library's first
            nl.build(d, n, box, g["morse"][3], g["skin"], stream=s)
            compute_morse_gpu(d, f, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), n, box,
                              MorseParams.make(*g["morse"]), precision=precision, stream=s)
        s.synchronize()
        assert rel_rms(f.double().cpu().numpy(), fo) < (FP64_TOL if precision == "fp64"
                                                        else MIXED_FORCE_TOL)
