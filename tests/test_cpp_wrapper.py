"""The header-only C++ layer (include/tdmd_b200.hpp) compiles in both of the
reference's precision modes, links against the C ABI library, and its
host-side calls (config, setfl tables, Nose-Hoover chain, errors) give the
reference's values.  No GPU needed."""
from __future__ import annotations

import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(tmp_path, define):
    from tdmd_claude_b200 import _lib
    so = _lib.LIB_PATH
    gxx = shutil.which("g++")
    if gxx is None or not os.path.isdir(os.path.join(CUDA_HOME, "include")):
        pytest.skip("no host C++ compiler or CUDA headers")
    exe = str(tmp_path / f"wrapper_{define}")
    cmd = [gxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", f"-D{define}",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA_HOME, "include"),
           os.path.join(ROOT, "tests", "cpp", "wrapper_host.cpp"), "-o", exe,
           so, f"-Wl,-rpath,{os.path.dirname(so)}",
           "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


@pytest.mark.parametrize("define,precision", [("TDMD_PRECISION_FP64", 0),
                                              ("TDMD_PRECISION_MIXED", 1)])
def test_cpp_layer_host_calls(tmp_path, define, precision):
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    setfl = str(tmp_path / "cu.eam.alloy")
    TIO.write_setfl(setfl, W.cu_eam_tables())
    s = W.morse_256()
    data = str(tmp_path / "c0.data")
    TIO.write_lammps_data(data, s)
    exe = _build(tmp_path, define)
    out = subprocess.run([exe, setfl, data, str(tmp_path / "out")], check=True,
                         capture_output=True, text=True).stdout
    kv = dict(line.split(" ", 1) for line in out.strip().splitlines())
    assert int(kv["precision"]) == precision
    assert int(kv["rebuild"]) == 10 and abs(float(kv["skin"]) - 0.3) < 1e-7
    assert int(kv["ntypes"]) == 1 and abs(float(kv["cutoff"]) - 5.0) < 1e-6
    ref = golden("ref_nhc.json")["cases"][0]["scale"][0]
    tol = 0.0 if precision == 0 else 1e-7  # the mixed build returns a float
    assert abs(float(kv["scale0"]) - ref) <= tol
    assert float(kv["t_target"]) == 400.0
    # masses are `real` as in the reference's SystemState: float in the mixed build
    m1 = float(s.masses[1]) if precision == 0 else float(np.float32(s.masses[1]))
    assert int(kv["natoms"]) == 256 and float(kv["mass1"]) == m1
    assert float(kv["x0"]) == float(s.positions[0, 0])
    assert int(kv["data_roundtrip"]) == 1
    assert int(kv["dump_n"]) == 256 and float(kv["dump_fx0"]) == 1.5 and int(kv["dump_id0"]) == 1
    assert abs(float(kv["setfl_cutoff"]) - 5.0) < 1e-6
    assert int(kv["error"]) == 9  # TDMD_ERR_IO: the setfl file cannot be opened
