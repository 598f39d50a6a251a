"""The GPU-backed tdmd_standalone (tdmd_claude_b200/bin) run as a VerifyLab
script runs the reference binary: a subprocess with the reference's flags,
thermo lines parsed with a "Step N  PE  KE  TE  T" pattern, the step-0 force
dump read back.  Step-0 PE and forces equal the reference's (FP64 1e-10
relative, mixed 1e-5 RMS); NVE total energy stays flat."""
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
BIN = {"fp64": os.path.join(ROOT, "tdmd_claude_b200", "bin", "tdmd_standalone"),
       "mixed": os.path.join(ROOT, "tdmd_claude_b200", "bin", "tdmd_standalone_mixed")}
THERMO = re.compile(r"^Step\s+(\d+)\s+PE\s+(\S+)\s+KE\s+(\S+)\s+TE\s+(\S+)\s+T\s+(\S+)", re.M)


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


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_standalone_cli_matches_reference(cuda, tmp_path, precision):
    from tdmd_claude_b200 import io as TIO
    data, g = _data_file(tmp_path)
    dump = str(tmp_path / "f0.dump")
    final = str(tmp_path / "final.dump")
    morse = ",".join(str(x) for x in g["morse"])
    out = subprocess.run([sys.executable, BIN[precision], "--data", data, "--nsteps", "200",
                          "--thermo", "50", "--morse", morse, "--skin", str(g["skin"]),
                          "--dump-forces", dump, "--dump-final", final],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    rows = [tuple(float(x) for x in m) for m in THERMO.findall(out.stdout)]
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
    assert "Neighbor list rebuilds:" in out.stdout

