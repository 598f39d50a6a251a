"""The GPU-backed tdmd_standalone run as a VerifyLab script runs the
reference binary: a subprocess with the reference's flags, thermo lines
parsed with a "Step N  PE  KE  TE  T" pattern, the step-0 force dump read
back.  Two drivers: the native C++ one (tdmd_claude_b200/bin/native, built
against include/tdmd_b200.hpp per precision as the reference's binary is)
and the Python one (tdmd_claude_b200/bin).  Step-0 PE and forces equal the
reference's (FP64 1e-10 relative, mixed 1e-5 RMS); NVE total energy stays
flat; both drivers print the same thermo lines and dumps."""
from __future__ import annotations

import os
import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import golden, rel_rms

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = {("python", "fp64"): [sys.executable,
                            os.path.join(ROOT, "tdmd_claude_b200", "bin", "tdmd_standalone")],
       ("python", "mixed"): [sys.executable,
                             os.path.join(ROOT, "tdmd_claude_b200", "bin",
                                          "tdmd_standalone_mixed")],
       ("native", "fp64"): [os.path.join(ROOT, "tdmd_claude_b200", "bin", "native",
                                         "tdmd_standalone")],
       ("native", "mixed"): [os.path.join(ROOT, "tdmd_claude_b200", "bin", "native",
                                          "tdmd_standalone_mixed")]}
THERMO = re.compile(r"^Step\s+(\d+)\s+PE\s+(\S+)\s+KE\s+(\S+)\s+TE\s+(\S+)\s+T\s+(\S+)", re.M)


def _run(driver, precision, args):
    cmd = BIN[(driver, precision)]
    assert os.path.exists(cmd[-1]), f"{cmd[-1]} missing: build the library first"
    out = subprocess.run(cmd + args, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    return out.stdout


def _data_file(tmp_path):
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    g = golden("ref_morse_256.json")
    s = W.morse_256()
    s.positions = np.array(g["positions"])
    s.velocities = np.array(g["velocities"])
    path = str(tmp_path / "cu256.data")
    TIO.write_lammps_data(path, s)
    return path, g


@pytest.mark.parametrize("driver", ["native", "python"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_standalone_cli_matches_reference(cuda, tmp_path, driver, precision):
    from tdmd_claude_b200 import io as TIO
    data, g = _data_file(tmp_path)
    dump = str(tmp_path / "f0.dump")
    final = str(tmp_path / "final.dump")
    morse = ",".join(str(x) for x in g["morse"])
    stdout = _run(driver, precision, ["--data", data, "--nsteps", "200", "--thermo", "50",
                                      "--morse", morse, "--skin", str(g["skin"]),
                                      "--dump-forces", dump, "--dump-final", final])
    rows = [tuple(float(x) for x in m) for m in THERMO.findall(stdout)]
    steps = [int(r[0]) for r in rows]
    assert steps[:5] == [0, 50, 100, 150, 200] and steps[-1] == 200   # + the "Final:" line
    pe0 = rows[0][1]
    tol = 1e-10 if precision == "fp64" else 1e-6
    assert abs(pe0 - g["reference_pe"]) <= tol * abs(g["reference_pe"])
    te = np.array([r[3] for r in rows])
    assert np.abs(te - te[0]).max() / 256 < 1e-3   # Morse has no shift at rc
    ids, types, pos, forces = TIO.read_force_dump(dump)
    assert np.array_equal(ids, np.arange(1, 257))
    assert rel_rms(forces, np.array(g["reference_forces"])) < (1e-10 if precision == "fp64"
                                                                 else 1e-5)
    ids, _, pos_final, _ = TIO.read_force_dump(final)
    assert pos_final.shape == (256, 3)
    assert "Neighbor list rebuilds:" in stdout


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_native_and_python_drivers_agree_eam(cuda, tmp_path, precision):
    """Ternary EAM (864 atoms, three element types) through both drivers.
    FP64: the same thermo lines and dumps, bit for bit.  Mixed: the native
    binary holds masses in `real` (float) as the reference's mixed build
    does, the Python driver in double, so the step-0 PE and forces are equal
    and the rest agrees to the float rounding of the masses."""
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    s = W.ternary(6)
    data = str(tmp_path / "ternary.data")
    setfl = str(tmp_path / "ternary.eam.alloy")
    TIO.write_lammps_data(data, s)
    TIO.write_setfl(setfl, W.ternary_eam_tables())
    res = {}
    for driver in ("native", "python"):
        d0, d1 = str(tmp_path / f"{driver}0.dump"), str(tmp_path / f"{driver}1.dump")
        stdout = _run(driver, precision, ["--data", data, "--eam", setfl, "--nsteps", "60",
                                          "--thermo", "20", "--skin", "0.5",
                                          "--dump-forces", d0, "--dump-final", d1])
        res[driver] = (THERMO.findall(stdout), TIO.read_force_dump(d0), TIO.read_force_dump(d1))
    (tn, f0n, f1n), (tp, f0p, f1p) = res["native"], res["python"]
    assert len(tn) == len(tp) == 5  # steps 0, 20, 40, 60 and the "Final:" line
    assert [r[0] for r in tn] == [r[0] for r in tp]
    assert tn[0][1] == tp[0][1]  # step-0 PE: positions and the potential only
    for x, y in zip(f0n, f0p):  # step-0 dump: ids, types, positions, forces
        assert np.array_equal(x, y)
    if precision == "fp64":
        assert tn == tp
        for x, y in zip(f1n, f1p):
            assert np.array_equal(x, y)
    else:
        a = np.array([[float(v) for v in r[1:4]] for r in tn])
        b = np.array([[float(v) for v in r[1:4]] for r in tp])
        assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max()
        assert np.array_equal(f1n[0], f1p[0])
        assert np.abs(f1n[2] - f1p[2]).max() < 1e-6
