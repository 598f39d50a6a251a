"""Pins the CPU oracle (oracle/tdmd_oracle.c) to the reference's golden
vectors and to the reference's own CPU path.  CPU only."""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from conftest import golden


def test_two_atoms_morse_analytic(oracle):
    """VerifyLab two-atoms-morse: U and F at r = 2.5 (tolerance 1e-14)."""
    g = golden("two_atoms_morse.json")
    p = g["potential"]
    pos = np.array([a["pos_A"] for a in g["atoms"]], np.float64)
    pe, f, _ = oracle.morse_forces(pos, (-50, -50, -50), (50, 50, 50), p["D0_eV"],
                                   p["alpha_inv_A"], p["r0_A"], p["cutoff_A"], 0.0)
    assert abs(pe - g["step0"]["U_eV"]) < 1e-14
    f1 = np.array(g["step0"]["force_on_atom_1_eV_per_A"])
    assert np.abs(f[0] - f1).max() / abs(f1[0]) < 1e-14
    assert np.abs(f[1] + f1).max() / abs(f1[0]) < 1e-14


def test_morse_equilibrium(oracle):
    """U(r0) = -D, F(r0) = 0 (test_morse.cpp:39-47)."""
    pos = np.array([[0, 0, 0], [2.866, 0, 0]], np.float64)
    pe, f, _ = oracle.morse_forces(pos, (-20,) * 3, (20,) * 3, 0.3429, 1.3588, 2.866, 6.0, 0.0)
    assert abs(pe + 0.3429) < 1e-15
    assert np.abs(f).max() < 1e-15


def test_run0_morse_lammps(oracle):
    """256-atom perfect lattice vs the LAMMPS run-0 dump (max |dF| 1e-12) and
    the reference CPU PE."""
    g = golden("run0_morse_256.json")
    pos = np.array(g["positions"])
    D, a, r0, rc = g["morse"]
    pe, f, _ = oracle.morse_forces(pos, g["lo"], g["hi"], D, a, r0, rc, g["skin"])
    assert np.abs(f - np.array(g["lammps_forces"])).max() < g["tolerance_fp64"]
    assert pe == g["reference_pe"]
    assert abs(pe - g["lammps_pe"]) / abs(g["lammps_pe"]) < 1e-7


def test_run0_eam_lammps(oracle, mishin_setfl):
    g = golden("run0_eam_256.json")
    eam = oracle.OracleEam.from_setfl(mishin_setfl)
    m = golden("run0_morse_256.json")
    pos = np.array(m["positions"])
    r = eam.forces(pos, np.ones(len(pos), np.int32), m["lo"], m["hi"], g["skin"])
    assert np.abs(r["forces"] - np.array(g["lammps_forces"])).max() < g["tolerance_fp64"]
    assert r["pe"] == g["reference_pe"]
    # FCC bulk cohesive energy of this potential (test_eam.cpp:398-415)
    assert abs(r["pe"] / len(pos) + 3.54) < 0.1


def test_reference_morse_jitter(oracle):
    """Jittered 256-atom Cu, rc 6.0 + skin 0.3: bit-equal to the reference."""
    g = golden("ref_morse_256.json")
    pos = np.array(g["positions"])
    pe, f, _ = oracle.morse_forces(pos, g["lo"], g["hi"], *g["morse"], g["skin"])
    assert pe == g["reference_pe"]
    assert np.array_equal(f, np.array(g["reference_forces"]))


def test_reference_half_list_and_cells(oracle):
    g = golden("ref_morse_256.json")
    pos = np.array(g["positions"])
    c, o, nb = oracle.neighbor_list(pos, g["lo"], g["hi"], 6.0, g["skin"], half=True)
    assert nb.size == g["half_list"]["total"]
    assert np.array_equal(c, g["half_list"]["counts"])
    assert np.array_equal(nb, g["half_list"]["neighbors"])
    nc, cc, co, ca, _ = oracle.cell_list(pos, g["lo"], g["hi"], 6.3)
    assert np.array_equal(nc, g["cell_list"]["nc"])
    assert np.array_equal(cc, g["cell_list"]["counts"])
    assert np.array_equal(co, g["cell_list"]["offsets"])
    assert np.array_equal(ca, g["cell_list"]["atoms"])


def test_full_list_is_half_list_union_transpose(oracle):
    """Full list = half list + its transpose (test_device_neighbor_list.cu:78-128)."""
    g = golden("ref_morse_256.json")
    pos = np.array(g["positions"])
    ch, oh, nh = oracle.neighbor_list(pos, g["lo"], g["hi"], 6.0, 0.3, half=True)
    cf, of, nf = oracle.neighbor_list(pos, g["lo"], g["hi"], 6.0, 0.3, half=False)
    assert nf.size == 2 * nh.size
    n = len(pos)
    full = [set(nf[of[i]:of[i] + cf[i]]) for i in range(n)]
    exp = [set() for _ in range(n)]
    for i in range(n):
        for j in nh[oh[i]:oh[i] + ch[i]]:
            exp[i].add(int(j))
            exp[int(j)].add(i)
    assert full == exp


def _write_eam(tmpdir):
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    t = W.cu_eam_tables()
    p = os.path.join(tmpdir, "cu.eam.alloy")
    TIO.write_setfl(p, t)
    return p, t


def test_reference_eam_analytic(oracle):
    g = golden("ref_eam_256.json")
    m = golden("ref_morse_256.json")
    with tempfile.TemporaryDirectory() as d:
        p, t = _write_eam(d)
        eam = oracle.OracleEam.from_setfl(p)
    for key, v in g["coeffs"].items():
        kind, idx = (int(x) for x in key.split("_"))
        c = eam.coeffs(kind, idx)
        assert np.array_equal(c[v["index"]], v["values"])
    pos = np.array(m["positions"])
    r = eam.forces(pos, np.ones(len(pos), np.int32), m["lo"], m["hi"], g["skin"])
    assert r["pe"] == g["reference_pe"]
    assert np.array_equal(r["forces"], np.array(g["reference_forces"]))


def test_nhc_matches_reference(oracle):
    g = golden("ref_nhc.json")
    for c in g["cases"]:
        M = c["chain"]
        st = np.zeros(3 * M)
        oracle.lib().orc_nhc_init(st, M, c["t_target"], c["t_period"], c["n_dof"])
        got = [oracle.lib().orc_nhc_half_step(st, M, c["t_target"], c["t_period"], c["n_dof"],
                                              c["dt"], ke) for ke in c["ke"]]
        assert got == c["scale"]


def test_md_matches_reference_cpu_loop(oracle):
    """100 NVE steps: the oracle's plain VV loop (CPU driver order) equals the
    reference CPU loop bit for bit."""
    g = golden("ref_morse_256.json")
    pos = np.array(g["positions"])
    vel = np.array(g["velocities"])
    masses = np.array(g["masses"])
    n = len(pos)
    types = np.ones(n, np.int32)
    L = oracle.lib()
    b = oracle.make_box(g["lo"], g["hi"])
    f = np.zeros((n, 3))
    D, a, r0, rc = g["morse"]
    c, o, nb = oracle.neighbor_list(pos, g["lo"], g["hi"], rc, g["skin"], half=True)
    L.orc_morse_forces(pos.reshape(-1), n, C.byref(b), D, a, r0, rc, c, o, nb, f.reshape(-1),
                       np.zeros(6))
    since = 0
    for _ in range(100):
        L.orc_half_kick(vel.reshape(-1), f.reshape(-1), types, masses, n, 0.001)
        L.orc_drift(pos.reshape(-1), vel.reshape(-1), n, 0.001, C.byref(b))
        since += 1
        if since >= 10:
            c, o, nb = oracle.neighbor_list(pos, g["lo"], g["hi"], rc, g["skin"], half=True)
            since = 0
        pe = L.orc_morse_forces(pos.reshape(-1), n, C.byref(b), D, a, r0, rc, c, o, nb,
                                f.reshape(-1), np.zeros(6))
        L.orc_half_kick(vel.reshape(-1), f.reshape(-1), types, masses, n, 0.001)
    assert np.array_equal(pos, np.array(g["md100"]["positions"]))
    assert np.array_equal(vel, np.array(g["md100"]["velocities"]))
    assert pe == g["md100"]["pe"]


def test_fast_path_md_close_to_cpu_loop(oracle):
    """The scheduler restatement (fused kicks, single-image wrap) stays
    within rounding of the CPU loop over 100 steps."""
    g = golden("ref_morse_256.json")
    r = oracle.md_run(np.array(g["positions"]), np.array(g["velocities"]),
                      np.ones(256, np.int32), np.array(g["masses"]), g["lo"], g["hi"], 0.001,
                      g["skin"], 10, [100], morse=g["morse"])
    dp = r["pos"] - np.array(g["md100"]["positions"])
    L = np.array(g["hi"]) - np.array(g["lo"])
    dp -= np.round(dp / L) * L
    assert np.abs(dp).max() < 1e-11
    assert np.abs(r["vel"] - np.array(g["md100"]["velocities"])).max() < 1e-9


def test_reference_harness_equals_oracle_on_random_gas(oracle, ref_lib):
    """Random gas with atoms at exact skin boundaries (test_neighbor_list.cpp)."""
    rng = np.random.default_rng(7)
    L = 20.0
    pos = rng.uniform(0, L, size=(400, 3))
    pos[1] = pos[0] + np.array([6.3, 0, 0])  # exactly at r_list
    pos[1] %= L
    per = np.ones(3, np.int32)
    lo, hi = np.zeros(3), np.full(3, L)
    n = len(pos)
    cnt, off = np.zeros(n, np.int32), np.zeros(n, np.int32)
    nb = np.zeros(200 * n, np.int32)
    tot = ref_lib.ref_half_list(pos.reshape(-1), n, lo, hi, per, 6.0, 0.3, cnt, off, nb, 200 * n)
    c, o, nbo = oracle.neighbor_list(pos, lo, hi, 6.0, 0.3, half=True)
    assert tot == nbo.size and np.array_equal(c, cnt) and np.array_equal(nbo, nb[:tot])
