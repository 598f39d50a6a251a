"""The C-ABI library without a GPU: it loads, exports every symbol the header
declares, and its host-only entry points (setfl parsing, spline
coefficients, NHC chain, argument checks) agree with the oracle."""
from __future__ import annotations

import os
import re
import tempfile

import numpy as np
import pytest

from conftest import ROOT, golden


@pytest.fixture(scope="module")
def L():
    from tdmd_claude_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from tdmd_claude_b200 import build
        build.build()
    return _lib.lib()


def header_symbols():
    with open(os.path.join(ROOT, "include", "tdmd_b200.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(tdmd_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol(L):
    from tdmd_claude_b200 import _lib
    syms = header_symbols()
    assert len(syms) > 40
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_lib.SIGNATURES), set(syms) ^ set(_lib.SIGNATURES)
    assert L.tdmd_abi_version() == 2


def test_config_defaults_follow_reference(L):
    from tdmd_claude_b200 import make_config
    c = make_config()
    assert (c.dt, c.r_skin, c.rebuild_every) == (0.001, 1.0, 10)   # FastPipelineConfig
    assert (c.t_period, c.nhc_length) == (0.1, 3)                   # NHCConfig
    assert (c.dt_max, c.dt_min, c.c2) == (0.002, 0.0001, 0.05)     # PipelineConfig


def _setfl(tmp):
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    t = W.cu_eam_tables()
    p = os.path.join(tmp, "cu.eam.alloy")
    TIO.write_setfl(p, t)
    return p, t


def test_setfl_reader_and_splines_equal_oracle(L, oracle):
    from tdmd_claude_b200 import EamAlloy
    g = golden("ref_eam_256.json")
    with tempfile.TemporaryDirectory() as d:
        p, t = _setfl(d)
        e = EamAlloy().read_setfl(p)
        oe = oracle.OracleEam.from_setfl(p)
    info = e.info()
    assert (info["ntypes"], info["nrho"], info["nr"], info["cutoff"]) == (1, 2000, 2000, 5.0)
    for kind in (0, 1, 2):
        assert np.array_equal(e.coeffs(kind, 0), oe.coeffs(kind, 0))
    for key, v in g["coeffs"].items():
        kind, idx = (int(x) for x in key.split("_"))
        assert np.array_equal(e.coeffs(kind, idx)[v["index"]], v["values"])


def test_eam_from_tables_equals_setfl(L):
    from tdmd_claude_b200 import EamAlloy
    with tempfile.TemporaryDirectory() as d:
        p, t = _setfl(d)
        a = EamAlloy().read_setfl(p)
    b = EamAlloy.from_tables(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    for kind in (0, 1, 2):
        np.testing.assert_allclose(a.coeffs(kind, 0), b.coeffs(kind, 0), rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("contents", [
    "",                                                       # RejectEmptyFile
    "# line 1\n# line 2\n# line 3\n",                         # RejectCommentsOnly
    "# c1\n# c2\n# c3\n1 Cu\n500 0.01 500 0.012 6.0\n29 63.546 3.615 fcc\n",
    "# c1\n# c2\n# c3\n1 Cu\n500 0.01 500 0.012 6.0\n29 63.546 3.615 fcc\n" + "0.0\n" * 10,
    "# c1\n# c2\n# c3\n1 Cu\n50 0.01 50 0.012 0.6\n29 63.546 3.615 fcc\n" + "-1.0\n" * 50
    + "0.5\n" * 50,                                           # RejectMissingPairBlock
])
def test_malformed_setfl_rejected(L, contents):
    """test_eam.cpp:451-508: malformed setfl files raise (here TDMD_ERR_PARSE)."""
    from tdmd_claude_b200 import EamAlloy, TdmdError
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "bad.eam.alloy")
        with open(p, "w") as f:
            f.write(contents)
        with pytest.raises(TdmdError) as ei:
            EamAlloy().read_setfl(p)
    assert ei.value.code == 4


def test_missing_setfl_file(L):
    from tdmd_claude_b200 import EamAlloy, TdmdError
    with pytest.raises(TdmdError):
        EamAlloy().read_setfl("/nonexistent/file.eam.alloy")


def test_nhc_host_chain_equals_reference(L):
    from tdmd_claude_b200 import NoseHooverChain
    g = golden("ref_nhc.json")
    for c in g["cases"]:
        h = NoseHooverChain(c["t_target"], c["t_period"], c["chain"], c["dt"], c["n_dof"])
        got = [h.half_step(ke) for ke in c["ke"]]
        np.testing.assert_allclose(got, c["scale"], rtol=1e-15, atol=0)


def test_null_and_range_arguments(L):
    import ctypes as C
    from tdmd_claude_b200 import _lib
    assert L.tdmd_eam_read_setfl(None, None) == 1
    assert L.tdmd_eam_create(0, 10, 0.1, 10, 0.1, 1.0, None, None, None, None) == 1
    h = C.c_void_p()
    assert L.tdmd_nhc_create(300.0, 0.1, 99, 0.001, 3, C.byref(h)) == 1
    assert b"chain" in L.tdmd_last_error()
    assert L.tdmd_sched_run_until(None, 3) == 1
    assert _lib.STATUS_NAMES[6] == "NLIST_OVERFLOW"


def test_workload_generators():
    from tdmd_claude_b200 import workloads as W
    s = W.eam_131k()
    assert s.n == 131072 and s.lo == (0.0, 0.0, 0.0) and abs(s.hi[0] - 115.68) < 1e-12
    ke = 0.5 * (s.masses[s.types] * W.MVV2E * (s.velocities ** 2).sum(1)).sum()
    T = 2 * ke / ((3 * s.n - 3) * W.KB)
    assert abs(T - 300.0) < 1e-9
    assert np.abs((s.masses[s.types][:, None] * s.velocities).sum(0)).max() < 1e-6
    assert (s.positions >= 0).all() and (s.positions < 115.68).all()
    t = W.ternary(4)
    assert set(np.unique(t.types)) == {1, 2, 3}


def test_lammps_data_roundtrip():
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    s = W.morse_256()
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "c0.data")
        TIO.write_lammps_data(p, s)
        r = TIO.read_lammps_data(p)
    assert np.array_equal(r.positions, s.positions)
    assert np.array_equal(r.velocities, s.velocities)
    assert np.array_equal(r.types, s.types) and np.array_equal(r.masses, s.masses)


def test_reference_reads_our_data_file(ref_lib):
    """The reference's read_lammps_data parses what io.write_lammps_data writes."""
    import ctypes as C
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    s = W.morse_256()
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "c0.data")
        TIO.write_lammps_data(p, s)
        n, nt = C.c_int64(), C.c_int32()
        lo, hi = np.zeros(3), np.zeros(3)
        pos, vel = np.zeros((256, 3)), np.zeros((256, 3))
        ty, ids, m = np.zeros(256, np.int32), np.zeros(256, np.int32), np.zeros(2)
        assert ref_lib.ref_read_data(p.encode(), C.byref(n), C.byref(nt), lo, hi, pos.ctypes.data,
                                     vel.ctypes.data, ty.ctypes.data, ids.ctypes.data,
                                     m.ctypes.data) == 0
    assert np.array_equal(pos, s.positions) and np.array_equal(vel, s.velocities)


def test_batch_rejects_thermostat_and_bad_boxes(L):
    import ctypes as C
    from tdmd_claude_b200 import Box, MorseParams, make_config
    boxes = (Box * 1)(Box.make((0, 0, 0), (20, 20, 20)))
    natoms = (C.c_int32 * 1)(10)
    p = MorseParams.make(0.3429, 1.3588, 2.866, 6.0)
    h = C.c_void_p()
    cfg = make_config(t_target=300.0)
    assert L.tdmd_batch_create_morse(1, boxes, natoms, C.byref(p), C.byref(cfg),
                                     C.byref(h)) == 8      # TDMD_ERR_UNSUPPORTED
    small = (Box * 1)(Box.make((0, 0, 0), (10, 10, 10)))    # edge < 2 (rc + skin)
    assert L.tdmd_batch_create_morse(1, small, natoms, C.byref(p), C.byref(make_config()),
                                     C.byref(h)) == 1      # TDMD_ERR_INVALID_ARGUMENT
    assert L.tdmd_batch_create_morse(0, boxes, natoms, C.byref(p), C.byref(make_config()),
                                     C.byref(h)) == 1


def test_fit_rejects_bad_arguments(L):
    import ctypes as C
    from tdmd_claude_b200 import Box
    box = Box.make((0, 0, 0), (20, 20, 20))
    pos = np.zeros((1, 2, 3))
    pos[0, 1, 0] = 2.5
    typ = np.ones(2, np.int32)
    h = C.c_void_p()
    p, t = pos.ctypes.data_as(C.c_void_p), typ.ctypes.data_as(C.c_void_p)
    assert L.tdmd_fit_create(0, 2, C.byref(box), p, t, 5.0, 0, C.byref(h)) == 1
    assert L.tdmd_fit_create(1, 2, C.byref(box), p, t, -1.0, 0, C.byref(h)) == 1
    assert L.tdmd_fit_create(1, 2, C.byref(box), p, t, 5.0, 7, C.byref(h)) == 1
    small = Box.make((0, 0, 0), (8, 8, 8))               # edge < 2 cutoff
    assert L.tdmd_fit_create(1, 2, C.byref(small), p, t, 5.0, 0, C.byref(h)) == 1


def test_standalone_banner_usage_and_argument_errors():
    """The tdmd_standalone command line (no GPU needed for these paths)."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "tdmd_claude_b200", "bin", "tdmd_standalone")
    run = lambda *a: subprocess.run([sys.executable, exe, *a], capture_output=True,  # noqa: E731
                                    text=True, timeout=120)
    out = run("--help")
    assert out.returncode == 0 and "--data <file>" in out.stdout
    out = run()
    assert out.returncode == 0 and "Use --data <file>" in out.stdout
    out = run("--morse", "1,2")
    assert out.returncode == 1 and "D,alpha,r0,rc" in out.stderr
    out = run("--precision", "fp16")
    assert out.returncode == 1


def test_two_element_setfl_parses():
    """A written two-element setfl reads back with ntypes 2, its cutoff and
    the embedding and density splines passing through the tabulated values
    (test_eam.cpp:163-170)."""
    import os
    import tempfile

    from conftest import two_element_tables

    from tdmd_claude_b200 import EamAlloy
    from tdmd_claude_b200 import io as TIO
    t = two_element_tables()
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "ab.eam.alloy")
        TIO.write_setfl(p, t, comment="two-element test alloy")
        eam = EamAlloy().read_setfl(p)
    assert eam.ntypes() == 2 and abs(eam.cutoff() - 6.0) < 1e-12
    # the a coefficients of F and rho are the tabulated values (phi is
    # built from r phi / r, so it is not compared here)
    for kind, tab in ((0, t.F), (1, t.rho)):
        for k in range(2):
            c = eam.coeffs(kind, k)
            n = len(c) // 4
            assert np.allclose(c[:n], tab[k][:n], rtol=1e-14, atol=1e-14), (kind, k)
