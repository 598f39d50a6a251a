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
    assert L.tdmd_abi_version() == 3


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


def test_eam_from_phi_samples_equals_setfl_tables(L):
    """tdmd_eam_create_sampled: tables given as phi(r) samples (r*phi / r,
    phi(0) = 0, as the reference's EamAlloy stores them) build the same
    splines as the r*phi arrays of the setfl, bit for bit (ternary: six
    pair tables)."""
    from tdmd_claude_b200 import EamAlloy
    from tdmd_claude_b200 import workloads as W
    t = W.ternary_eam_tables()
    a = EamAlloy.from_tables(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    rphi = np.asarray(t.rphi, np.float64).reshape(-1, t.nr)
    r = np.arange(t.nr) * t.dr
    phi = np.zeros_like(rphi)
    phi[:, 1:] = rphi[:, 1:] / r[1:]
    b = EamAlloy.from_samples(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, phi)
    npairs = t.ntypes * (t.ntypes + 1) // 2
    for kind, count in ((0, t.ntypes), (1, t.ntypes), (2, npairs)):
        for idx in range(count):
            assert np.array_equal(a.coeffs(kind, idx), b.coeffs(kind, idx))


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


def test_missing_files_are_io_errors(L, tmp_path):
    """A file that cannot be opened is TDMD_ERR_IO for every reader and
    writer (LammpsDataReader.FileNotFound, tests/unit/test_lammps_data_reader.cpp)."""
    from tdmd_claude_b200 import EamAlloy, TdmdError
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    missing = str(tmp_path / "no_such_dir" / "file")
    for call in (lambda: EamAlloy().read_setfl(missing + ".eam.alloy"),
                 lambda: TIO.read_lammps_data(missing + ".data"),
                 lambda: TIO.read_force_dump(missing + ".dump"),
                 lambda: TIO.write_lammps_data(missing + ".data", W.morse_256())):
        with pytest.raises(TdmdError) as ei:
            call()
        assert ei.value.code == 9 and "cannot open" in str(ei.value)


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


# ---------------------------------------------------------------------------
# Native file formats (tdmd_read_lammps_data & co.) against the reference's
# own readers, compiled from its sources into oracle/_ref.
# ---------------------------------------------------------------------------
def _ref_read(ref_lib, path):
    import ctypes as C
    n, nt = C.c_int64(), C.c_int32()
    lo, hi = np.zeros(3), np.zeros(3)
    assert ref_lib.ref_read_data(path.encode(), C.byref(n), C.byref(nt), lo, hi, None, None,
                                 None, None, None) == 0
    N = n.value
    pos, vel = np.zeros((N, 3)), np.zeros((N, 3))
    ty, ids, m = np.zeros(N, np.int32), np.zeros(N, np.int32), np.zeros(nt.value + 1)
    assert ref_lib.ref_read_data(path.encode(), C.byref(n), C.byref(nt), lo, hi,
                                 pos.ctypes.data, vel.ctypes.data, ty.ctypes.data,
                                 ids.ctypes.data, m.ctypes.data) == 0
    return pos, vel, ty, ids, m, lo, hi


def _data_files(tmp):
    """The reference's own data fixtures (where its tree is present) and a
    file written here with velocities, blank lines inside sections and a
    comment after the Atoms keyword."""
    from conftest import REF_TREE
    out = []
    if REF_TREE is not None:
        for f in ("tests/data/cu_fcc_256.data", "tests/data/cu_fcc_32.data",
                  "tests/data/4atoms.data"):
            p = os.path.join(REF_TREE, f)
            if os.path.exists(p):
                out.append(p)
    p = os.path.join(tmp, "odd.data")
    with open(p, "w") as f:
        f.write("odd layout\n\n3 atoms\n2 atom types\n\n0 10 xlo xhi\n-1 9 ylo yhi\n"
                "0.5 7.5 zlo zhi\n\nMasses\n\n1 63.546\n\n2 58.69\n\nAtoms # atomic\n\n"
                "3 2 1.25 2.5 3.75\n1 1 0.1 0.2 0.3\n\n2 1 4 5 6\n\nVelocities\n\n"
                "2 0.5 -0.5 0.25\n1 1e-3 2e-3 3e-3\n3 -1 -2 -3\n")
    out.append(p)
    return out


def test_native_data_reader_equals_reference(L, ref_lib, tmp_path):
    """tdmd_read_lammps_data gives the reference read_lammps_data's arrays
    (lammps_data_reader.cpp:33-204), bit for bit."""
    from tdmd_claude_b200 import io as TIO
    for p in _data_files(str(tmp_path)):
        s = TIO.read_lammps_data(p)
        pos, vel, ty, ids, m, lo, hi = _ref_read(ref_lib, p)
        assert np.array_equal(s.positions, pos), p
        assert np.array_equal(s.velocities, vel), p
        assert np.array_equal(s.types, ty) and np.array_equal(s.ids, ids), p
        assert np.array_equal(s.masses, m), p
        assert np.array_equal(s.lo, lo) and np.array_equal(s.hi, hi), p


def test_native_data_roundtrip_and_reference_reads_it(L, ref_lib, tmp_path):
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    s = W.ternary(3, seed=5)
    p = str(tmp_path / "t.data")
    TIO.write_lammps_data(p, s)
    r = TIO.read_lammps_data(p)
    for a, b in ((r.positions, s.positions), (r.velocities, s.velocities), (r.types, s.types),
                 (r.ids, s.ids), (r.masses, s.masses)):
        assert np.array_equal(a, b)
    pos, vel, ty, ids, m, lo, hi = _ref_read(ref_lib, p)
    assert np.array_equal(pos, s.positions) and np.array_equal(vel, s.velocities)
    assert np.array_equal(ty, s.types) and np.array_equal(m, s.masses)


@pytest.mark.parametrize("body,what", [
    ("t\n\n2 atoms\n1 atom types\n0 1 xlo xhi\n0 1 ylo yhi\n\nAtoms\n\n1 1 0 0 0\n2 1 0 0 0\n",
     "incomplete box"),
    ("t\n\n2 atoms\n1 atom types\n0 1 xlo xhi\n0 1 ylo yhi\n0 1 zlo zhi\n\nAtoms\n\n1 1 0 0 0\n",
     "premature end"),
    ("t\n\n2 atoms\n1 atom types\n0 1 xlo xhi\n0 1 ylo yhi\n0 1 zlo zhi\n\nAtoms\n\n"
     "1 1 0 0 0\n2 1 0 x 0\n", "bad Atoms line"),
    ("t\n\n2 atoms\n1 atom types\n0 1 xlo xhi\n0 1 ylo yhi\n0 1 zlo zhi\n\nAtoms\n\n"
     "1 1 0 0 0\n7 1 0 0 0\n", "out of range"),
    ("t\n\n2 atoms\n1 atom types\n0 1 xlo xhi\n0 1 ylo yhi\n0 1 zlo zhi\n\nMasses\n\n1 2.0\n",
     "no Atoms section"),
    ("t\n\n0 atoms\n", "invalid atom count"),
])
def test_native_data_reader_rejects_malformed(L, tmp_path, body, what):
    from tdmd_claude_b200 import TdmdError
    from tdmd_claude_b200 import io as TIO
    p = str(tmp_path / "bad.data")
    with open(p, "w") as f:
        f.write(body)
    with pytest.raises(TdmdError) as ei:
        TIO.read_lammps_data(p)
    assert ei.value.code == 4 and what in str(ei.value)


def test_native_force_dump_roundtrip_and_reference_dump(L, tmp_path):
    """Dumps written natively read back exactly (17 digits; float forces
    widened exactly); the reference's committed LAMMPS dump reads into the
    values of the golden fixture made from it."""
    from conftest import REF_TREE
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    s = W.morse_256()
    rng = np.random.default_rng(1)
    for dt in (np.float64, np.float32):
        f = rng.standard_normal((s.n, 3)).astype(dt)
        p = str(tmp_path / f"d_{np.dtype(dt).name}.dump")
        # shuffled ids: the reader sorts by id
        perm = rng.permutation(s.n)
        sp = W.System(s.positions[perm], s.velocities[perm], s.types[perm], s.ids[perm],
                      s.masses, s.lo, s.hi)
        TIO.write_force_dump(p, sp, f[perm], step=42)
        ids, ty, pos, fr = TIO.read_force_dump(p)
        assert np.array_equal(ids, s.ids) and np.array_equal(ty, s.types)
        assert np.array_equal(pos, s.positions) and np.array_equal(fr, f.astype(np.float64))
        with open(p) as fh:
            assert fh.read().startswith("ITEM: TIMESTEP\n42\nITEM: NUMBER OF ATOMS\n256\n")
    if REF_TREE is not None:
        p = os.path.join(REF_TREE, "verifylab/cases/run0-force-match/forces_morse.dump")
        if os.path.exists(p):
            ids, ty, pos, fr = TIO.read_force_dump(p)
            assert np.array_equal(fr, np.array(golden("run0_morse_256.json")["lammps_forces"]))


def test_native_setfl_writer_roundtrip(L, mishin_setfl, tmp_path):
    """A read setfl written back natively reads again to the same tables and
    spline coefficients (the Mishin Cu file), and the reference's
    EamAlloy::read_setfl reads the written file to the same forces."""
    from tdmd_claude_b200 import EamAlloy
    from tdmd_claude_b200 import io as TIO
    a = EamAlloy().read_setfl(mishin_setfl)
    p = str(tmp_path / "again.eam.alloy")
    TIO.write_eam_setfl(p, a)
    b = EamAlloy().read_setfl(p)
    assert a.info() == b.info()
    for kind in (0, 1, 2):
        assert np.array_equal(a.coeffs(kind, 0), b.coeffs(kind, 0))
    with open(p) as f, open(mishin_setfl) as g:
        assert f.readline() == g.readline()      # comment lines kept
    from oracle import oracle as O
    R = O.ref()
    if R is not None:
        import ctypes as C
        m = golden("run0_morse_256.json")
        pos = np.array(m["positions"])
        out = []
        for path in (mishin_setfl, p):
            h = R.ref_eam_load(path.encode())
            f = np.zeros_like(pos)
            pe = R.ref_eam_forces(h, pos.reshape(-1), np.ones(256, np.int32), 256,
                                  np.array(m["lo"]), np.array(m["hi"]), np.ones(3, np.int32),
                                  1.0, f.reshape(-1))
            R.ref_eam_free(h)
            out.append((pe, f))
        assert out[0][0] == out[1][0] and np.array_equal(out[0][1], out[1][1])
        _ = C


def test_reference_data_reader_unit_test(L):
    """The reference's own LammpsDataReader unit test
    (tests/unit/test_lammps_data_reader.cpp: Basic4Atoms, FileNotFound),
    compiled unchanged against this library's native reader
    (`make -C oracle reftests`), on its 4-atom input (tests/golden/4atoms.data,
    copied from the reference by make_golden.py)."""
    import subprocess
    exe = os.path.join(ROOT, "oracle", "_ref", "reftest_test_lammps_data_reader_fp64")
    if not os.path.exists(exe):
        pytest.skip("reference unit tests not built (make -C oracle reftests)")
    env = dict(os.environ, TDMD_TEST_DATA_DIR=os.path.join(ROOT, "tests", "golden"))
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120, env=env)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "[       OK ] LammpsDataReader.Basic4Atoms" in out.stdout
    assert "[       OK ] LammpsDataReader.FileNotFound" in out.stdout


@pytest.mark.parametrize("name,tests", [
    ("test_zone_partition", ("ZonePartition.EveryAtomInExactlyOneZone",
                             "ZonePartition.AtomsInCorrectZone", "ZonePartition.ZoneNeighbors")),
    ("test_zone_state_machine", ("ZoneStateMachine.LegalTransitions",
                                 "ZoneStateMachine.IllegalTransitions",
                                 "ZoneStateMachine.TimeStepMonotonicity")),
])
def test_reference_zone_unit_tests(L, tmp_path, name, tests):
    """The reference's zone tests (tests/unit/test_zone_partition.cpp,
    test_zone_state_machine.cpp) compiled unchanged against the C++ layer's
    own single-rank zone types (`make -C oracle reftests`), on the
    reference's 256-atom data file (from the run0_morse_256.json fixture)."""
    import subprocess
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    exe = os.path.join(ROOT, "oracle", "_ref", f"reftest_{name}_own")
    if not os.path.exists(exe):
        pytest.skip("reference unit tests not built (make -C oracle reftests)")
    g = golden("run0_morse_256.json")
    pos = np.array(g["positions"])
    n = len(pos)
    TIO.write_lammps_data(str(tmp_path / "cu_fcc_256.data"),
                          W.System(pos, np.zeros_like(pos), np.ones(n, np.int32),
                                   np.arange(1, n + 1, dtype=np.int32), np.array(g["masses"]),
                                   tuple(g["lo"]), tuple(g["hi"])))
    env = dict(os.environ, TDMD_TEST_DATA_DIR=str(tmp_path))
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120, env=env)
    assert out.returncode == 0, out.stdout + out.stderr
    for t in tests:
        assert f"[       OK ] {t}" in out.stdout
